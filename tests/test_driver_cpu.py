"""TTC's driver surface on the host: argument parsing, names, index fusion, the generated shim (compiled
with nvcc, not run), and the tuning database (round trip, corrupt file)."""
import sqlite3
import subprocess
from pathlib import Path

import pytest

import oracle.ttc_ref as ref
from ttc_b200 import TTCError, sql_util, ttc, ttc_util

ROOT = Path(__file__).resolve().parent.parent


def test_parse_args_matches_ttc_flags():
    a = ttc.parse_args(["--perm=1,0,2", "--size=1000,768,16", "--beta=1.0", "--dataType=zc", "--alpha=0.5",
                        "--lda=1000,770,16", "--maxImplementations=7", "--architecture=cuda", "--ignoreDatabase",
                        "--blockings=32x32,64x64", "--loopPerm=0,1,2-2,1,0", "--threadsPerBlock=256", "--noTest"])
    assert a.idxPerm == [1, 0, 2] and a.size == [1000, 768, 16]
    assert (a.floatTypeA, a.floatTypeB) == ("double complex", "float complex")
    assert a.alpha == 0.5 and a.beta == 1.0 and a.lda == [1000, 770, 16]
    assert a.maxNumImplementations == 7 and a.ignoreDatabase == 1 and a.noTest == 1
    assert a.blockings == [(32, 32), (64, 64)] and a.loopPermutations == [[0, 1, 2], [2, 1, 0]]
    assert a.architecture == "cuda"
    with pytest.raises(TTCError):
        ttc.parse_args(["--perm=1,0", "--size=3,4", "--bogus=1"])
    with pytest.raises(TTCError):
        ttc.parse_args(["--perm=1,0", "--size=3,4,5"])
    with pytest.raises(TTCError):
        ttc.parse_args(["--perm=1,0", "--size=3,4", "--dataType=q"])
    with pytest.raises(TTCError):
        ttc.parse_args(["--perm=1,0", "--size=3,4", "--threadsPerBlock=100"])


def test_transpose_names_follow_ttc():
    a = ttc_util.TTCargs([1, 0, 2], [1000, 768, 16])
    a.beta = 1.0
    assert ttc.getTransposeName(a) == "sCuTranspose_102_1000x768x16"
    a.beta = 0.0
    assert ttc.getTransposeName(a) == "sCuTranspose_102_1000x768x16_bz"
    a.floatTypeA, a.floatTypeB = "double complex", "float complex"
    assert ttc.getTransposeName(a) == "zsCuTranspose_102_1000x768x16_bz"   # TTC's own spelling
    assert ttc._function_name(a) == "zcCuTranspose_102_1000x768x16_bz"


def test_fuse_indices_mirror_matches_reference_restatement():
    import numpy as np
    rng = np.random.default_rng(4)
    for _ in range(200):
        r = int(rng.integers(1, 6))
        size = [int(x) for x in rng.integers(2, 6, r)]
        perm = [int(x) for x in rng.permutation(r)]
        s1, p1, l1, b1 = list(size), list(perm), [], []
        ttc_util.fuseIndices(s1, p1, [], l1, b1)
        # empty (dense) lda/ldb stay empty in the caller's lists, as in TTC (ttc_util.py:214-222)
        assert (l1, b1) == ([], [])
        l1, b1 = ttc_util.denseLeadingDims(s1, p1, l1, b1)
        s2, p2, l2, b2 = ref.fuse_indices(size, perm)
        assert (s1, p1, l1, b1) == (s2, p2, l2, b2)
        # explicit leading dimensions are fused in place
        s3, p3, l3, b3 = list(size), list(perm), list(size), [size[p] for p in perm]
        ttc_util.fuseIndices(s3, p3, [], l3, b3)
        assert (s3, p3, l3, b3) == (s2, p2, l2, b2)


def test_cost_loop_mirror():
    import numpy as np
    rng = np.random.default_rng(6)
    for _ in range(50):
        r = int(rng.integers(2, 6))
        size = [int(x) for x in rng.integers(2, 9, r)]
        perm = [int(x) for x in rng.permutation(r)]
        lp = [int(x) for x in rng.permutation(r)]
        assert ttc_util.getCostLoop(lp, perm, size) == ref.cost_loop(lp, perm, size)


@pytest.mark.parametrize("dtype,beta", [("s", 1.0), ("zc", 0.0), ("cz", 2.0), ("ds", 0.0)])
def test_generated_shim_compiles(tmp_path, dtype, beta):
    a = ttc_util.TTCargs([2, 0, 1], [7, 8, 9])
    a.floatTypeA, a.floatTypeB = ttc_util.TYPES_OF_PREFIX[dtype]
    a.beta = beta
    name = ttc.getTransposeName(a)
    h, src = ttc.emit_shim(a, name, ttc._function_name(a), {"tile_elems": 1024, "loop_order": 1}, [7, 8, 9],
                           [2, 0, 1], None, None)
    (tmp_path / f"{name}.h").write_text(h)
    (tmp_path / f"{name}.cu").write_text(src)
    r = subprocess.run(["/usr/local/cuda/bin/nvcc", "-c", "-I", str(ROOT / "include"), "-o", str(tmp_path / "x.o"),
                        str(tmp_path / f"{name}.cu")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    nm = subprocess.run(["nm", str(tmp_path / "x.o")], capture_output=True, text=True).stdout
    assert ttc._function_name(a) in nm and name in nm


def test_database_round_trip_and_corrupt_file(tmp_path):
    db = str(tmp_path / "ttc.db")
    variants = [{"tuning": {"tile_elems": 1024}, "bandwidth": 10.0, "time": 1e-3, "rank": 1},
                {"tuning": {"run_bytes": 256}, "bandwidth": 20.0, "time": 5e-4, "rank": 0}]
    sql_util.insert(db, [1000, 768, 16], [1, 0, 2], "float", "float", 1.0, 1.0, " NVIDIA B200", "h", variants, 1.0)
    hit = sql_util.lookup(db, [1000, 768, 16], [1, 0, 2], "float", "float", 1.0, " NVIDIA B200")
    assert hit["tuning"] == {"run_bytes": 256} and hit["bandwidth"] == 20.0
    assert sql_util.lookup(db, [1000, 768, 16], [1, 0, 2], "float", "float", 0.0, " NVIDIA B200") is None
    assert sql_util.lookup(db, [1000, 768, 16], [1, 0, 2], "double", "double", 1.0, " NVIDIA B200") is None
    con = sqlite3.connect(db)
    rows = con.execute("SELECT * FROM fastest0Percent").fetchall()
    assert len(rows) == 1
    con.close()
    bad = tmp_path / "bad.db"
    bad.write_bytes(b"this is not a database" * 100)
    with pytest.raises(sql_util.DatabaseUnavailable):
        sql_util.lookup(str(bad), [4, 4], [1, 0], "float", "float", 0.0, "x")


def test_main_reports_errors_without_exiting(capsys):
    assert ttc.main(["--perm=1,0", "--size=3,4", "--lda=2,4", "--architecture=cuda"]) == 1
    out = capsys.readouterr().out
    assert "leading dimension of A" in out


def test_loop_perm_flags_become_explicit_rasters():
    """--loopPerm restricts the search to the given loop orders, each kept as given (the explicit
    raster, ttcb_tuning loop_order 4); without it, TTC's cost-ranked orders join the presets."""
    from ttc_b200.autotune import Problem, candidate_tunings
    a = ttc.parse_args(["--perm=1,0,2", "--size=1000,768,16", "--loopPerm=2,0,1-1,2,0"])
    space = ttc._tunings_from_args(a, "s")
    assert space["loop_order"] == [] and space["rasters"] == [[2, 0, 1], [1, 2, 0]]
    cands = candidate_tunings(Problem([1, 0, 2], [1000, 768, 16], "s"), 1000, space)
    rasters = {tuple(t["raster"]) for t in cands if "raster" in t}
    assert rasters == {(2, 0, 1), (1, 2, 0)}
    assert all("raster" in t for t in cands)
    b = ttc.parse_args(["--perm=1,0,2", "--size=1000,768,16"])
    assert ttc._tunings_from_args(b, "s")["rasters"] == ("ttc", 2)


def test_report_summarises_the_fastest_variants_per_rank(tmp_path, capsys):
    """TTC's benchmark summary (generatePlots.py:141-265) over the fastest0Percent view: per rank the
    bandwidth range of the fastest variants and their speedup over the reference bandwidth."""
    from ttc_b200 import report
    db = str(tmp_path / "ttc.db")
    v = lambda bw: [{"tuning": {}, "bandwidth": bw, "time": 1e-3, "rank": 0},
                    {"tuning": {"run_bytes": 128}, "bandwidth": bw / 2, "time": 2e-3, "rank": 1}]
    sql_util.insert(db, [100, 200, 30], [1, 0, 2], "float", "float", 1.0, 0.0, "dev", "h", v(100.0), 1.0, 50.0)
    sql_util.insert(db, [10, 20, 30], [2, 1, 0], "float", "float", 1.0, 0.0, "dev", "h", v(300.0), 1.0, 100.0)
    sql_util.insert(db, [64, 64], [1, 0], "double", "double", 1.0, 0.0, "dev", "h", v(40.0), 1.0)
    rows = report.benchmark_summary(db)
    assert [r["dim"] for r in rows] == [2, 3]
    r3 = rows[1]
    assert (r3["count"], r3["bw_min"], r3["bw_max"], r3["bw_avg"]) == (2, 100.0, 300.0, 200.0)
    assert (r3["speedup_min"], r3["speedup_max"]) == (2.0, 3.0)
    assert rows[0]["speedup_count"] == 0  # no reference bandwidth recorded
    out = tmp_path / "s.csv"
    assert report.main(["--db", db, "--csv", str(out)]) == 0
    assert "avg GiB/s" in capsys.readouterr().out and out.read_text().startswith("dim,count")
    assert report.benchmark_summary(db, "floatTypeA = 'double'")[0]["count"] == 1


def test_cpu_architecture_runs_ttcs_own_generator(tmp_path, monkeypatch, capsys):
    """--architecture=avx goes, with the same flags, to TTC's own CPU driver (ttc.py:1132-1376) from a
    TTC checkout: it generates, compiles, checks and times its variants and writes the header; without
    a checkout the request fails with a message instead of silently running on the GPU."""
    from oracle.make_ref import DEFAULT_SOURCE
    from pathlib import Path
    argv = ["--perm=1,0,2", "--size=64,48,5", "--architecture=avx", "--compiler=g++", "--maxImplementations=2",
            "--numThreads=2", "--ignoreDatabase"]
    monkeypatch.chdir(tmp_path)
    monkeypatch.setenv("TTC_SOURCE_DIR", str(tmp_path / "nowhere"))
    assert ttc.main(argv) == 1
    assert "TTC_SOURCE_DIR" in capsys.readouterr().out
    if not (Path(DEFAULT_SOURCE) / "ttc" / "ttc.py").exists():
        pytest.skip("the TTC sources are not on this machine")
    monkeypatch.setenv("TTC_SOURCE_DIR", DEFAULT_SOURCE)
    name, gibps = ttc.generateTransposition(ttc.parse_args(argv))
    assert gibps > 0 and (tmp_path / "ttc_transpositions" / f"{name}.h").exists()
    assert "implementations done" in capsys.readouterr().out
