"""The C-ABI library loads without a GPU and exports what include/sopb.h
declares, with the structure layouts the bindings assume."""
import ctypes
import os
import re
import subprocess

import pytest

import sopb

REPO = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HEADER = os.path.join(REPO, "include", "sopb.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sopb_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "sopb_run" in names and "sopb_job_create" in names and len(names) >= 18


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    lib = sopb.lib()
    assert hasattr(lib, name), name


def test_struct_layout_matches_c(tmp_path):
    # every field of the ctypes mirrors at the C compiler's offset
    fields = [("sopb_params", sopb.Params, f[0]) for f in sopb.Params._fields_]
    fields += [("sopb_job_desc", sopb.JobDesc, f[0]) for f in sopb.JobDesc._fields_]
    body = "".join('printf("%%zu\\n", offsetof(%s, %s));' % (c, f) for c, _, f in fields)
    prog = tmp_path / "layout.c"
    prog.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "sopb.h"\n'
        'int main(void){printf("%zu\\n%zu\\n", sizeof(sopb_params), sizeof(sopb_job_desc));' + body +
        ' return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(REPO, "include"), str(prog), "-o", str(exe)])
    vals = [int(v) for v in subprocess.check_output([str(exe)]).split()]
    want = [ctypes.sizeof(sopb.Params), ctypes.sizeof(sopb.JobDesc)] + [getattr(t, f).offset for _, t, f in fields]
    assert vals == want


def test_default_params_are_reference_defaults():
    p = sopb.default_params()
    # PARAMETER() defaults: langevin.h:13-14, covalent.h:12-13, pairs.h:12-15,
    # pairlist.h:12-14, possiblepairlist.h:12-13, gsop.h:34, pulling.h:17,
    # indentation.h:24-35, bdhitea.h:17-21
    expect = dict(zeta=50.0, temperature=0.6, kspring_cov=20.0, R_limit=2.0, a=3.8, el=1.0, pairs_cutoff=20.0,
                  pairlist_cutoff=20.0, pairs_freq=1000, pairs_threshold=200.0, possiblepairs_freq=100000,
                  max_pairs=512, max_possiblePairs=4096, nav=1000, k_trans=0.05, indentationTipZeta=5000.0,
                  indentationTipB=1.0, indentationSurfB=1.0, indentationRetractionStep=-1, hi_a=1.8,
                  hi_capricious=1, hi_unlisted=1, hi_epsmax=999.0)
    for k, v in expect.items():
        assert getattr(p, k) == pytest.approx(v, rel=1e-7), k


def test_status_strings():
    for code in range(10):
        assert sopb.lib().sopb_status_string(code)
    assert b"capacity" in sopb.lib().sopb_status_string(sopb.ERR_CAPACITY)


def test_invalid_arguments_are_status_codes():
    lib = sopb.lib()
    assert lib.sopb_run(None, None, 0, 1) == sopb.ERR_INVALID
    assert lib.sopb_job_destroy(None) == sopb.ERR_INVALID
    assert lib.sopb_generate_seeds(1, -1, None) == sopb.ERR_INVALID


def test_context_without_device_reports_nodevice():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert sopb.lib().sopb_context_create(0, None, ctypes.byref(h)) == sopb.ERR_NODEVICE


def test_oracle_defaults_equal_library_defaults():
    """The CPU baseline fills its job descriptions from the oracle's own
    table of the reference's PARAMETER() defaults; it must equal the
    library's sopb_default_params field for field."""
    import oracle_py
    a = sopb.params_dict(oracle_py.default_params())
    b = sopb.params_dict(sopb.default_params())
    assert a == b
