"""Host-side logic of libxbtrav.so and its C ABI (CPU only, no compute calls on a GPU)."""
import numpy as np
import pytest

import xbtrav


def test_library_exports_every_declared_symbol():
    L = xbtrav.lib()
    names = xbtrav.declared_symbols()
    assert "xb_traverse" in names and "xb_ctx_create" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.xb_abi_version() == 3


def test_status_strings():
    L = xbtrav.lib()
    for s in (0, -1, -2, -3, -4, -5, -6, -7, -8):
        assert L.xb_status_str(s)
    assert L.xb_status_str(-99) == b"unknown status"


def _check_clean_csr(ro, ci):
    n = len(ro) - 1
    assert ro[0] == 0 and (np.diff(ro) >= 0).all()
    assert ((ci >= 0) & (ci < n)).all()
    src = np.repeat(np.arange(n), np.diff(ro))
    assert (src != ci).all(), "self loop"
    for v in range(0, n, max(1, n // 64)):
        nb = ci[ro[v]:ro[v + 1]]
        assert (np.diff(nb) > 0).all(), "unsorted or duplicate adjacency"
    # symmetric: (u,v) present iff (v,u) present
    key = src.astype(np.int64) * n + ci
    rkey = ci.astype(np.int64) * n + src
    assert np.array_equal(np.sort(key), np.sort(rkey))


def test_rmat_generator_is_clean_deterministic_and_thread_independent():
    a = xbtrav.HostCSR.rmat(12, 8, seed=7, threads=1)
    b = xbtrav.HostCSR.rmat(12, 8, seed=7, threads=5)
    c = xbtrav.HostCSR.rmat(12, 8, seed=8, threads=3)
    ra, ca = a.arrays()
    rb, cb = b.arrays()
    rc, cc = c.arrays()
    assert np.array_equal(ra, rb) and np.array_equal(ca, cb)
    assert not np.array_equal(ca[: len(cc)], cc[: len(ca)])
    _check_clean_csr(ra, ca)


def test_rmat16_shape_matches_the_configured_recipe():
    # R-MAT scale 16 / edge factor 16, a/b/c = .57/.19/.19: ~1.82M directed entries,
    # ~18.8k isolated vertices, max degree ~9.8k.
    g = xbtrav.HostCSR.rmat(16, 16, seed=0x5EED)
    inf = g.info()
    assert inf["n"] == 65536
    assert 1_750_000 < inf["m"] < 1_900_000
    assert 17_000 < inf["isolated"] < 20_500
    assert 8_000 < inf["max_degree"] < 12_000


def test_er_generator():
    g = xbtrav.HostCSR.er(5000, 12000, seed=3)
    ro, ci = g.arrays()
    assert len(ro) == 5001
    _check_clean_csr(ro, ci)
    assert 2 * 12000 * 0.98 < len(ci) <= 2 * 12000


def test_source_selection():
    g = xbtrav.HostCSR.rmat(10, 4, seed=11)
    ro, ci = g.arrays()
    deg = np.diff(ro)
    s1 = xbtrav.select_sources_csr(ro, 99, 100)
    s2 = xbtrav.select_sources_csr(ro, 99, 100)
    s3 = xbtrav.select_sources_csr(ro, 98, 100)
    assert np.array_equal(s1, s2) and not np.array_equal(s1, s3)
    assert len(np.unique(s1)) == 100
    assert (deg[s1] > 0).all()
    with pytest.raises(xbtrav.XbError) as e:
        xbtrav.select_sources_csr(ro, 1, int((deg > 0).sum()) + 1)
    assert e.value.status == xbtrav.XB_ERR_ARG
    assert len(xbtrav.select_sources_csr(ro, 1, 0)) == 0


def test_text_format_round_trip(tmp_path):
    g = xbtrav.HostCSR.rmat(8, 4, seed=5)
    ro, ci = g.arrays()
    rp, cp = str(tmp_path / "row_offsets.txt"), str(tmp_path / "col_indices.txt")
    g.save_text(rp, cp)
    # the reference format: one integer per line
    lines = open(rp).read().split("\n")
    assert lines[0] == "0" and int(lines[len(ro) - 1]) == ro[-1]
    h = xbtrav.HostCSR.load_text(rp, cp)
    r2, c2 = h.arrays()
    assert np.array_equal(ro, r2) and np.array_equal(ci, c2)


def test_text_load_errors(tmp_path):
    with pytest.raises(xbtrav.XbError) as e:
        xbtrav.HostCSR.load_text(str(tmp_path / "nope"), str(tmp_path / "nope2"))
    assert e.value.status == xbtrav.XB_ERR_IO
    rp, cp = tmp_path / "r.txt", tmp_path / "c.txt"
    rp.write_text("0\n2\n3\n")
    cp.write_text("1\n")  # last offset says 3 entries, file has 1
    with pytest.raises(xbtrav.XbError) as e:
        xbtrav.HostCSR.load_text(str(rp), str(cp))
    assert e.value.status == xbtrav.XB_ERR_IO
    cp.write_text("1\nx\n0\n")
    with pytest.raises(xbtrav.XbError):
        xbtrav.HostCSR.load_text(str(rp), str(cp))


def test_from_arrays_validation():
    with pytest.raises(xbtrav.XbError):
        xbtrav.HostCSR.from_arrays([0, 1, 2], [1, 5])  # id out of range
    with pytest.raises(xbtrav.XbError):
        xbtrav.HostCSR.from_arrays([0, 2, 1], [1, 0])  # decreasing offsets
    g = xbtrav.HostCSR.from_arrays([0, 1, 2], [1, 0])
    assert g.info()["n"] == 2


def test_declared_symbols_parse_every_header():
    names = xbtrav.declared_symbols()
    assert len(names) == len(set(names))
    assert all(n.startswith("xb_") for n in names)


def test_context_without_device_reports_nodev():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(xbtrav.XbError) as e:
        xbtrav.Context(0)
    assert e.value.status == xbtrav.XB_ERR_NODEV


def _build_example(tmp_path, name="example_traverse"):
    import os
    import subprocess

    import xbtrav as X

    pkg = os.path.dirname(X.LIB_PATH)
    root = os.path.dirname(pkg)
    exe = str(tmp_path / name)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(root, "include"), "-I", os.path.join(pkg, "host"),
                    os.path.join(pkg, "host", name + ".cpp"), "-L", pkg, "-lxbtrav",
                    f"-Wl,-rpath,{pkg}", "-o", exe], check=True)
    return exe


def test_runner_cli_compiles_and_parses_flags(tmp_path):
    """xbtrav_run takes the reference runners' gflags-style flags; usage and
    flag errors need no GPU."""
    import subprocess

    exe = _build_example(tmp_path, "xbtrav_run")
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--row_offsets" in r.stderr and "--path_buffer_ratio" in r.stderr
    assert subprocess.run([exe], capture_output=True, text=True).returncode == 2
    assert subprocess.run([exe, "--rmat=8:4", "--mode=bogus"], capture_output=True, text=True).returncode == 2
    # a full command line of the reference runner reaches the device step (no GPU here: a clean error)
    r = subprocess.run([exe, "--dataset=Tiny", "--rmat", "8:4", "--rounds=3", "--num_threads=4",
                        "--path_buffer_ratio=2", "--max_cuda_sms=0"], capture_output=True, text=True)
    assert "Run xbtrav (match) on Dataset Tiny" in r.stdout and r.returncode == 1 and "xbtrav error" in r.stderr


def test_cpp_host_api_compiles_and_links(tmp_path):
    import subprocess

    exe = _build_example(tmp_path)
    # usage error path runs without a GPU
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
