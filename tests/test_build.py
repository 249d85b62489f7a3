"""The in-tree build driver's user flags (CPU; nvcc and the linker faked).

KMY_NVCC_FLAGS adds nvcc flags to every unit (for example IEEE division in
the fused FP64 stages); a change of those flags must rebuild every unit, and
an unchanged set must rebuild none.
"""
import types

from kamayan_b200 import build as B


def test_user_flags_parse(monkeypatch):
    monkeypatch.setenv("KMY_NVCC_FLAGS", "-DSLAB_F64_NR=0  -DKMY_F64_NR=0")
    assert B.user_flags() == ["-DSLAB_F64_NR=0", "-DKMY_F64_NR=0"]
    monkeypatch.delenv("KMY_NVCC_FLAGS")
    assert B.user_flags() == []


def test_flag_change_rebuilds_every_unit(monkeypatch, tmp_path):
    srcs = [tmp_path / "a.cu", tmp_path / "b.cu"]
    compiled = []

    def fake_compile(src, verbose_ptxas=False, force=False):
        obj = B.BUILD / (src.stem + ".o")
        if force or not obj.exists():
            obj.write_text(" ".join(B.user_flags()))
            compiled.append(src.stem)
        return obj

    def fake_run(cmd, **kw):
        B.LIB.write_text("lib")
        return types.SimpleNamespace(returncode=0, stdout="", stderr="")

    monkeypatch.setattr(B, "BUILD", tmp_path / "_build")
    monkeypatch.setattr(B, "LIBDIR", tmp_path / "lib")
    monkeypatch.setattr(B, "LIB", tmp_path / "lib" / "libkmy_hydro.so")
    monkeypatch.setattr(B, "sources", lambda: srcs)
    monkeypatch.setattr(B, "compile_one", fake_compile)
    monkeypatch.setattr(B, "nvcc", lambda: "nvcc")
    monkeypatch.setattr(B.subprocess, "run", fake_run)

    monkeypatch.delenv("KMY_NVCC_FLAGS", raising=False)
    B.build(jobs=1)
    assert sorted(compiled) == ["a", "b"]
    compiled.clear()
    B.build(jobs=1)
    assert compiled == []
    monkeypatch.setenv("KMY_NVCC_FLAGS", "-DKMY_F64_NR=0")
    B.build(jobs=1)
    assert sorted(compiled) == ["a", "b"]
    assert (B.BUILD / "user_flags.txt").read_text() == "-DKMY_F64_NR=0"
    compiled.clear()
    B.build(jobs=1)
    assert compiled == []
    monkeypatch.delenv("KMY_NVCC_FLAGS")
    B.build(jobs=1)
    assert sorted(compiled) == ["a", "b"]
