"""Host-side logic of the product, no GPU: the C ABI library loads and
exports every declared symbol, the vite reader/writer, the reference-RGG
generator against the oracle and the reference's golden counts, the
Chung-Lu weight table against the oracle twin, and the CLI's argument
checks (main.cpp:238-275)."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import oracle
import xxtric_b200 as xt
from conftest import ROOT, load_fixtures, load_golden

GOLDEN = load_golden()
FIX = load_fixtures()
HEADER = os.path.join(ROOT, "include", "xtric.h")
CLI = os.path.join(ROOT, "xxtric_b200", "xtric")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(xt_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 20
    lib = xt.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding lists exactly the header's entry points
    assert set(names) == set(xt.EXPORTED), (set(names) ^ set(xt.EXPORTED))


def test_no_device_is_reported_not_faked():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(xt.XtError) as e:
        xt.Context(0)
    assert e.value.status == xt.XT_ERR_NO_DEVICE
    with pytest.raises(xt.XtError) as e:
        xt.Server(0)
    assert e.value.status == xt.XT_ERR_NO_DEVICE


def test_serve_estimate_is_linear_and_covers_the_build():
    # admission figure: grows with both sizes, adds up over a batch, and is
    # at least the bytes the builder's largest phase holds (8 B/row copied in,
    # 8 B/row union ids, 16 B/row keys, 40 B per unique edge while the
    # in-records are gathered)
    e = xt.serve_estimate
    assert e(-1, 0) < 0 and e(1, -1) < 0
    base = e(0, 0)
    assert 0 < base <= 8 << 20
    for nv, ne in [(1 << 10, 16 << 10), (1 << 20, 16 << 20), (3, 0)]:
        assert e(nv, ne) - base >= 72 * ne
        assert e(2 * nv, 2 * ne) - base == 2 * (e(nv, ne) - base)


@pytest.mark.parametrize("nprocs,radius", [(1, 0.0), (2, 0.0), (4, 0.0), (8, 0.0), (1, 0.03), (2, 0.02)])
def test_rgg_generator_matches_oracle(nprocs, radius):
    n = 4096
    off, tails = xt.generate_rgg(n, nprocs, radius)
    o_off, o_tails = oracle.ref_rgg(n, nprocs, radius)
    assert (off == o_off).all()
    assert (tails == o_tails).all()


@pytest.mark.parametrize("n", [1024, 4096, 16384, 65536])
def test_rgg_generator_reproduces_reference_graph(n):
    off, tails = xt.generate_rgg(n, 1)
    f = GOLDEN[f"rgg{n}"]
    assert len(tails) == f["directed_entries"]
    assert oracle.count_xxtric(off, tails) == f["triangles"]
    # rows sorted, symmetric, no self loops
    deg = np.diff(off)
    src = np.repeat(np.arange(n), deg)
    assert (src != tails).all()
    key = src * n + tails
    assert (np.diff(key) > 0).all()
    assert np.array_equal(np.sort(key), np.sort(tails * n + src))


def test_rgg_random_edges_deterministic():
    a = xt.generate_rgg(4096, 2, 0.0, 5.0, seed=3)
    b = xt.generate_rgg(4096, 2, 0.0, 5.0, seed=3)
    c = xt.generate_rgg(4096, 2, 0.0, 5.0, seed=4)
    base = xt.generate_rgg(4096, 2)
    assert (a[1] == b[1]).all()
    assert len(a[1]) > len(base[1])
    assert len(c[1]) != len(a[1]) or not (c[1] == a[1]).all()
    with pytest.raises(xt.XtError):
        xt.generate_rgg(4096, 2, 0.0, 100.0)
    with pytest.raises(xt.XtError):
        xt.generate_rgg(4096, 3)  # strip ranks must be a power of two


@pytest.mark.parametrize("elem", [8, 4])
def test_vite_roundtrip(tmp_path, elem):
    off, tails = xt.generate_rgg(1024, 1)
    p = str(tmp_path / "g.bin")
    xt.write_vite(p, off, tails, elem)
    assert os.path.getsize(p) == 2 * elem + (len(off)) * elem + len(tails) * 2 * elem
    o2, t2 = xt.read_vite(p, elem)
    assert (o2 == off).all() and (t2 == tails).all()


def test_vite_matches_reference_layout(tmp_path):
    # the layout graph.hpp:320-383 reads: header, offsets, {int64 tail, f64 weight}
    off, tails = xt.generate_rgg(1024, 1)
    p = str(tmp_path / "g.bin")
    xt.write_vite(p, off, tails)
    raw = np.fromfile(p, np.int64)
    assert raw[0] == 1024 and raw[1] == len(tails)
    assert (raw[2:2 + 1025] == off).all()
    rec = raw[2 + 1025:].reshape(-1, 2)
    assert (rec[:, 0] == tails).all()
    assert (rec[:, 1].view(np.float64) == 1.0).all()
    if os.path.exists(oracle.REF_TRIC):
        r = oracle.run_ref(["-f", p])
        assert r["triangles"] == GOLDEN["rgg1024"]["triangles"]


def test_vite_rejects_bad_files(tmp_path):
    off, tails = xt.generate_rgg(1024, 1)
    p = str(tmp_path / "g.bin")
    xt.write_vite(p, off, tails)
    data = open(p, "rb").read()
    open(p, "wb").write(data[:-8])  # truncated
    with pytest.raises(xt.XtError) as e:
        xt.read_vite(p)
    assert e.value.status == xt.XT_ERR_IO
    with pytest.raises(xt.XtError):
        xt.read_vite(str(tmp_path / "missing.bin"))
    bad = np.array([4, 2, 0, 1, 0, 2, 2], np.int64)  # offsets not monotone
    bad = np.concatenate([bad, np.array([1, 0, 0, 0], np.int64)])
    bad.tofile(p)
    with pytest.raises(xt.XtError):
        xt.read_vite(p)


def test_chunglu_cdf_matches_oracle():
    c1, m1 = xt.chunglu_cdf(1 << 16, 2.1, 64.0, 4096.0)
    c2, m2 = oracle.chunglu_cdf(1 << 16, 2.1, 64.0, 4096.0)
    assert m1 == m2
    assert (c1 == c2).all()
    w = np.diff(c1).astype(np.float64) / 1024.0
    assert abs(w.mean() - 64.0) < 3.0
    assert abs(w[0] - 4096.0) < 1.0


def run_cli(*args):
    return subprocess.run([CLI] + list(args), capture_output=True, text=True, timeout=120)


@pytest.mark.skipif(not os.path.exists(CLI), reason="xtric not built")
def test_cli_argument_errors():
    r = run_cli()
    assert r.returncode == 157 and "Must specify some options." in r.stderr
    r = run_cli("-l")  # the reference checks for an input first (main.cpp:253-257)
    assert r.returncode == 157 and "Must specify a binary file name" in r.stderr
    r = run_cli("-f", "x.bin", "-l")
    assert r.returncode == 157 and "Must specify -g for graph generation using LCG." in r.stderr
    r = run_cli("-f", "x.bin", "-p", "5")
    assert r.returncode == 157 and "add random edges" in r.stderr
    r = run_cli("-n", "1024", "-p", "150")
    assert r.returncode == 157 and "Invalid random edge percentage" in r.stderr
    r = run_cli("-f", "/nonexistent.bin")
    assert r.returncode == 157 and "Error opening file!" in r.stdout


def test_tsv_roundtrip_and_golden_count_input(tmp_path):
    # the amazon0302 fixture's rows (the reference's cuGraph TSV, ids as
    # given) written as TSV and read back: same rows, nv = largest id + 1
    src, dst = FIX["amazon0302_src"].astype(np.int32), FIX["amazon0302_dst"].astype(np.int32)
    p = str(tmp_path / "a.tsv")
    xt.write_tsv(p, src, dst)
    nv, s2, d2 = xt.read_tsv(p)
    assert nv == GOLDEN["amazon0302"]["nv"]
    assert (s2 == src).all() and (d2 == dst).all()
    off, tails = oracle.canon_csr(nv, s2.astype(np.int64), d2.astype(np.int64))
    assert oracle.count_merge(off, tails) == GOLDEN["amazon0302"]["triangles"]


def test_tsv_comments_weights_and_errors(tmp_path):
    p = tmp_path / "g.tsv"
    p.write_text("# a comment\n% another\n\n0\t1\t0.5\n1 2\n2\t0\t3\r\n")
    nv, s, d = xt.read_tsv(str(p))
    assert nv == 3 and s.tolist() == [0, 1, 2] and d.tolist() == [1, 2, 0]
    for bad in ("0\tx\n", "-1\t2\n", "0\n", "5\t99999999999\n"):
        p.write_text(bad)
        with pytest.raises(xt.XtError) as e:
            xt.read_tsv(str(p))
        assert e.value.status == xt.XT_ERR_IO
    with pytest.raises(xt.XtError) as e:
        xt.read_tsv(str(tmp_path / "missing.tsv"))
    assert e.value.status == xt.XT_ERR_IO


def compile_mirror_check(tmp_path):
    exe = str(tmp_path / "mirror_check")
    lib_dir = os.path.join(ROOT, "xxtric_b200")
    r = subprocess.run(["g++", "-O1", "-std=c++17", "-I", ROOT, "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "mirror_check.cpp"), "-o", exe, "-L", lib_dir,
                        "-lxtb200", "-Wl,-rpath," + lib_dir], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_mirror_compiles_and_reports_no_device(tmp_path):
    # the C++ mirror of the batch, per-edge and serving entry points builds
    # against the library; without a GPU it reports the library's status
    import torch
    exe = compile_mirror_check(tmp_path)
    if torch.cuda.is_available():
        pytest.skip("a GPU is present (the GPU test runs the program)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3 and r.stdout.startswith("error 9"), r.stdout


def test_bench_roofline_figures_come_from_the_committed_profiles():
    # the bench line's roofline.traffic is the DRAM bytes per full-size
    # k_count launch recorded in profiles/ (and its issue figure the small-case
    # capture's); they must parse and agree with the profiles' tables
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    t = bench.profiled_value("k_count_rmat_s24.md", "dram_bytes_per_launch_full_size")
    assert t is not None and 1e10 < t < 2e11
    text = open(os.path.join(ROOT, "profiles", "k_count_rmat_s24.md")).read()
    gb = float(re.search(r"dram__bytes_read\.sum \| ([0-9.]+) GB", text).group(1))
    assert abs(t / 1e9 - gb) < 0.1
    iss = bench.profiled_value("k_count_rmat_s22.md", "issue_slots_busy_frac")
    assert iss is not None and 0.0 < iss <= 1.0
    text = open(os.path.join(ROOT, "profiles", "k_count_rmat_s22.md")).read()
    pct = float(re.search(r"issue slots busy \| ([0-9.]+)%", text).group(1))
    assert abs(100 * iss - pct) < 0.1
    assert bench.profiled_value("no_such_profile.md", "dram_bytes_per_launch_full_size") is None
    # the roofline's basis: DRAM bytes over the kernel time when a capture exists
    class A:
        workload, scale = "rmat24", bench.SCALE
    info = {"alg_bytes": 171_750_000_000, "footprint_bytes": 6_800_000_000, "tail_alg_bytes": 744_750_000_000}
    r = bench.roofline_fields(A, info, 0.030)
    assert r["traffic"] == int(t) and abs(r["achieved"] - t / 0.030 / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12 and r["logical_frac"] > r["frac"]


def test_bench_reference_arm_loads_nothing_of_the_product(tmp_path):
    # the reference arm times the reference's own CPU path: it must not load
    # libxtb200.so (checked in a fresh interpreter, on the rgg sample, which
    # the oracle builds by itself)
    code = ("import sys, importlib.util; sys.argv=['bench.py']; "
            f"spec = importlib.util.spec_from_file_location('b', {os.path.join(ROOT, 'bench.py')!r}); "
            "b = importlib.util.module_from_spec(spec); spec.loader.exec_module(b); "
            "wl = b.Workload('rgg'); (off, tails), what, cfg = wl.cpu_sample(); "
            "import os; maps = open('/proc/self/maps').read(); "
            "print(len(tails), cfg['workload'][:20], 'libxtb200' in maps, 'xxtric_b200' in sys.modules)")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    n, *_, loaded, imported = r.stdout.split()
    assert int(n) > 0 and loaded == "False" and imported == "False"
