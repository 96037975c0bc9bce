"""The on-disk cubin cache of the run-time compiled block kernels
(KT_JIT_CACHE_DIR), on the host through kt_jit_compile_only (NVRTC, no GPU):

* a second compile of the same circuit's blocks loads the cubin from the
  directory instead of running NVRTC (kt_jit_cache_stats);
* a different circuit gets its own file;
* a file that fails its checks (truncated, or bytes changed) is compiled
  again and replaced, and the next compile loads it;
* a missing cache directory is created;
* without the variable nothing is read or written."""
from kettle_b200 import capi
from kettle_b200 import workloads as W


def _delta(before):
    now = capi.jit_cache_stats()
    return now["nvrtc_compiles"] - before["nvrtc_compiles"], now["disk_hits"] - before["disk_hits"]


def _files(d):
    return sorted(p for p in d.iterdir() if p.suffix == ".cubin")


def test_cubins_are_reused_checked_and_replaced(tmp_path, monkeypatch):
    monkeypatch.setenv("KT_JIT_CACHE_DIR", str(tmp_path))
    g = W.random_layers(14, 3, seed=5, mixed=True)

    s = capi.jit_cache_stats()
    assert capi.jit_compile_only(14, g) >= 1
    assert _delta(s) == (1, 0)
    files = _files(tmp_path)
    assert len(files) == 1
    good = files[0].read_bytes()

    s = capi.jit_cache_stats()
    assert capi.jit_compile_only(14, g) >= 1
    assert _delta(s) == (0, 1)

    # another circuit: another program, another file
    assert capi.jit_compile_only(14, W.random_layers(14, 3, seed=6, mixed=True)) >= 1
    assert len(_files(tmp_path)) == 2

    # a damaged file is compiled again and replaced by a good one
    for damaged in (good[: len(good) // 2], good[:-8] + bytes(8)):
        files[0].write_bytes(damaged)
        s = capi.jit_cache_stats()
        assert capi.jit_compile_only(14, g) >= 1
        assert _delta(s) == (1, 0)
        assert files[0].read_bytes() == good
        s = capi.jit_cache_stats()
        assert capi.jit_compile_only(14, g) >= 1
        assert _delta(s) == (0, 1)

    # no temporary files are left behind
    assert all(p.suffix == ".cubin" for p in tmp_path.iterdir())


def test_cache_directory_is_created(tmp_path, monkeypatch):
    d = tmp_path / "a" / "b"
    monkeypatch.setenv("KT_JIT_CACHE_DIR", str(d))
    assert capi.jit_compile_only(14, W.random_layers(14, 2, seed=8, mixed=True)) >= 1
    assert len(_files(d)) == 1


def test_no_cache_without_the_variable(tmp_path, monkeypatch):
    monkeypatch.delenv("KT_JIT_CACHE_DIR", raising=False)
    g = W.random_layers(14, 2, seed=7, mixed=True)
    s = capi.jit_cache_stats()
    assert capi.jit_compile_only(14, g) >= 1
    assert capi.jit_compile_only(14, g) >= 1
    assert _delta(s) == (2, 0)
    assert list(tmp_path.iterdir()) == []
    # an empty value is off too
    monkeypatch.setenv("KT_JIT_CACHE_DIR", "")
    s = capi.jit_cache_stats()
    assert capi.jit_compile_only(14, g) >= 1
    assert _delta(s) == (1, 0)
