"""The bench's hash of the CUDA code, which keys the ncu figures it reports:
comments and blank lines do not count, string literals (inline PTX) do."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_comments_do_not_count():
    a = 'int x = 1;  // one\n/* block\n comment */\nint y = 2;\n\n'
    b = 'int x = 1;\nint y = 2;  /* two */\n'
    assert bench.strip_comments(a) == bench.strip_comments(b) == "int x = 1;\nint y = 2;"


def test_string_literals_count():
    a = 'asm("mov.u64 %0, %%clock64; // not a comment" : "=l"(t));\nchar c = \'"\';'
    s = bench.strip_comments(a)
    assert "// not a comment" in s and "'\"'" in s
    assert bench.strip_comments('f("/*");\nint z;') == 'f("/*");\nint z;'


def test_code_change_changes_the_hash(tmp_path, monkeypatch):
    d = tmp_path / "sop-gpu_b200" / "csrc"
    d.mkdir(parents=True)
    (d / "k.cuh").write_text("int a = 1;  // note\n")
    monkeypatch.setattr(bench, "REPO", str(tmp_path))
    h0 = bench.source_hash()
    (d / "k.cuh").write_text("int a = 1;  // another note\n\n")
    assert bench.source_hash() == h0
    (d / "k.cuh").write_text("int a = 2;\n")
    assert bench.source_hash() != h0
