"""The drop-in `tpch_01` command line (the reference's flags in both spellings, src/main.cu:255-360,
README.md:47-58). Argument validation runs without a GPU; gpu-marked tests run the query and
compare the printed tables across data sources (generator, HBM residency, column cache)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tpchq01_gpu_b200", "bin", "tpch_01")


def run(args, cwd, timeout=300):
    return subprocess.run([BIN] + args, cwd=cwd, capture_output=True, text=True, timeout=timeout)


def tables(stdout):
    """The printed result blocks, one per run."""
    blocks, cur = [], None
    for line in stdout.splitlines():
        if line.startswith("Executing TPC-H Query 1"):
            if cur is not None:
                blocks.append(cur)
            cur = []
        elif cur is not None and "|" in line:
            cur.append(line.strip())
    if cur is not None:
        blocks.append(cur)
    return blocks


@pytest.mark.parametrize("args,needle", [
    (["--use-filter-pushdown"], "compression"),
    (["--threads-per-block=100"], "32"),
    (["--hash-table-placement=nowhere"], "kernel variant"),
    (["--no-such-flag"], "Unrecognized"),
    (["--sf=0"], "scale factor"),
])
def test_rejects_bad_arguments(tmp_path, args, needle):
    r = run(args, tmp_path)
    assert r.returncode != 0
    assert needle.lower() in (r.stderr + r.stdout).lower()


@pytest.mark.gpu
def test_spellings_residency_and_cache_agree(cuda, tmp_path):
    common = ["--apply-compression", "--print-results", "--rows=1000003", "--runs=2", "--seed=99"]
    outs = [
        run(common + ["--hash-table-placement=in-registers"], tmp_path),
        run(common + ["--hash-table-placement=in_registers_per_thread", "--resident"], tmp_path),
        run(common + ["--hash_table_placement=per-thread-shared-mem", "--use-filter-pushdown"], tmp_path),
        run(common + ["--use-coprocessing", "--cpu-fraction=0.3", "--streams=2"], tmp_path),
        run(common + ["--cache-dir=" + str(tmp_path / "cache"), "--write-cache"], tmp_path),
        run(common + ["--cache-dir=" + str(tmp_path / "cache"), "--resident"], tmp_path),
    ]
    for r in outs:
        assert r.returncode == 0, r.stderr
    ref = tables(outs[0].stdout)
    assert len(ref) == 2 and ref[0] and ref[0] == ref[1]
    for r in outs[1:]:
        assert tables(r.stdout) == ref
    assert os.path.exists(tmp_path / "results.csv")
    assert len(open(tmp_path / "results.csv").read().split()) == 2


@pytest.mark.gpu
def test_data_dir_layout_of_the_reference(cuda, tmp_path):
    """--data-dir=D reads D/<scale factor as std::to_string>/*.bin like the reference."""
    r = run(["--apply-compression", "--sf=0.01", "--data-dir=" + str(tmp_path / "data"), "--write-cache",
             "--runs=1"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert os.path.exists(tmp_path / "data" / "0.010000" / "shipdate.bin")


@pytest.mark.gpu
def test_tbl_path_of_the_reference(cuda, tmp_path):
    """Without a column cache, D/<sf>/lineitem.tbl is parsed (on the GPU) and the cache written,
    as the reference does (src/main.cu:441-475); the tables printed from the text, from the cache
    it left and from --tbl agree with the generator's."""
    common = ["--apply-compression", "--print-results", "--runs=1", "--sf=0.05", "--seed=7"]
    data = str(tmp_path / "data")
    made = run(common + ["--data-dir=" + data, "--write-tbl"], tmp_path)
    assert made.returncode == 0, made.stderr
    tbl = tmp_path / "data" / "0.050000" / "lineitem.tbl"
    assert tbl.exists() and not (tmp_path / "data" / "0.050000" / "shipdate.bin").exists()
    parsed = run(common + ["--data-dir=" + data], tmp_path)
    assert parsed.returncode == 0, parsed.stderr
    assert "Parsing the lineitem table" in parsed.stdout
    assert (tmp_path / "data" / "0.050000" / "shipdate.bin").exists()
    cached = run(common + ["--data-dir=" + data], tmp_path)
    direct = run(common + ["--tbl=" + str(tbl), "--resident"], tmp_path)
    generated = run(common, tmp_path)
    for r in (cached, direct, generated):
        assert r.returncode == 0, r.stderr
    ref = tables(generated.stdout)
    assert ref and ref[0]
    assert tables(made.stdout) == ref and tables(parsed.stdout) == ref
    assert tables(cached.stdout) == ref and tables(direct.stdout) == ref
