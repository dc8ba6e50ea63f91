"""The process boundary: the three CLI drivers and the dataset tools.

CPU: bin/cas_rmat_ones writes byte for byte what the reference's rmat_ones
(src/rmat_ones.c) wrote from the same edge list (tests/golden/rmat_ones);
bin/cas_gen writes the seeded generator's matrix; a driver with the wrong
argument count exits 1 as the reference's assert(argc == 2) ends it.

GPU: each driver on `cas_gen g500 12 8` prints the reference driver's lines
(tests/golden/driver_<algo>_g500_12_8.log, the reference's own stdout) —
the same CONFIGURATION line head, "<i>th run" lines with the five phase
times, the summary's keys in the reference's order and the same flop_cnt —
and its VERIFYRESULT triple (nnz, sum of columns, sum of values) equals the
reference's.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import casgemm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "contention-aware-spgemm_b200")
BIN = os.path.join(PKG, "bin")
GOLDEN = os.path.join(ROOT, "tests", "golden")
ALGOS = {"hash": "ams_hashspgemm", "hsersc": "ams_hserscspgemm", "hybacc": "ams_hybaccspgemm"}
RUN_LINE = re.compile(r"^(?:\x1b\[0;36m)?(\d+)th run\tinit_time: ([0-9.]+)\tsymb_time: ([0-9.]+)\t"
                      r"mgmt_time: ([0-9.]+)\tnumc_time: ([0-9.]+)\ttotal_time: ([0-9.]+)$")


@pytest.fixture(scope="module", autouse=True)
def built():
    need = [os.path.join(BIN, n) for n in list(ALGOS.values()) + ["cas_gen", "cas_rmat_ones"]]
    if not all(os.path.exists(p) for p in need):
        subprocess.run(["make", "-C", PKG, "drivers"], check=True, capture_output=True)


def summary_fields(text):
    line = [x for x in text.splitlines() if "dataset: " in x][-1]
    line = line.replace("\x1b[0;32m", "").replace("\x1b[0m", "")
    return [tuple(kv.split(": ", 1)) for kv in line.split("\t")]


def verify_triples(text):
    return [tuple(x.split("\t")[1:4]) for x in text.splitlines() if x.startswith("VERIFYRESULT:")]


def test_rmat_ones_matches_reference(tmp_path):
    ds = tmp_path / "dataset"
    ds.mkdir()
    shutil.copy(os.path.join(GOLDEN, "rmat_ones", "g500_4_2.txt"), ds)
    subprocess.run([os.path.join(BIN, "cas_rmat_ones"), "g500_4_2"], cwd=tmp_path, check=True, capture_output=True)
    for suffix in (".org.mtx", ".trs.mtx"):
        got = (ds / ("g500_4_2" + suffix)).read_bytes()
        want = open(os.path.join(GOLDEN, "rmat_ones", "g500_4_2" + suffix), "rb").read()
        assert got == want, suffix


def test_cas_gen_writes_the_generator_matrix(tmp_path):
    env = dict(os.environ, CAS_DATASET_DIR=str(tmp_path))
    subprocess.run([os.path.join(BIN, "cas_gen"), "g500", "8", "4"], check=True, capture_output=True, env=env)
    A = casgemm.gen_g500(8, 4, 8)
    for suffix in (".org.mtx", ".trs.mtx"):
        M = casgemm.mtx_read(str(tmp_path / ("g500_8_4" + suffix)))
        np.testing.assert_array_equal(M.row_ptrs, A.row_ptrs)
        np.testing.assert_array_equal(M.cols, A.cols)
    subprocess.run([os.path.join(BIN, "cas_gen"), "zipf", "z", "300", "900", "80", "2000", "5.0"], check=True,
                   capture_output=True, env=env)
    Z = casgemm.gen_zipf(300, 900, 80, 2000, 3, col_q=5.0)
    org = casgemm.mtx_read(str(tmp_path / "z.org.mtx"))
    trs = casgemm.mtx_read(str(tmp_path / "z.trs.mtx"))
    assert (org.to_scipy() != Z.to_scipy()).nnz == 0
    assert (trs.to_scipy() != Z.to_scipy().T).nnz == 0


@pytest.mark.parametrize("algo", sorted(ALGOS))
def test_driver_argument_count(algo):
    p = subprocess.run([os.path.join(BIN, ALGOS[algo])], capture_output=True, text=True)
    assert p.returncode == 1 and "usage" in p.stderr


def test_golden_logs_hold_the_reference_format():
    for algo in ALGOS:
        text = open(os.path.join(GOLDEN, f"driver_{algo}_g500_12_8.log")).read()
        assert text.startswith("CONFIGURATION:")
        runs = [RUN_LINE.match(x) for x in text.splitlines() if "th run" in x]
        assert len(runs) == 10 and all(runs)
        assert len(set(verify_triples(text))) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("algo", sorted(ALGOS))
def test_driver_matches_reference_log(tmp_path, algo):
    ds = tmp_path / "dataset"
    subprocess.run([os.path.join(BIN, "cas_gen"), "g500", "12", "8"], check=True, capture_output=True,
                   env=dict(os.environ, CAS_DATASET_DIR=str(ds)))
    env = dict(os.environ, CAS_RUN_NUM="3", CAS_VERIFY="1", CAS_CSR_CACHE="1")
    p = subprocess.run([os.path.join(BIN, ALGOS[algo]), "g500_12_8"], cwd=tmp_path, capture_output=True, text=True,
                       env=env, timeout=300)
    assert p.returncode == 0, p.stderr
    ref = open(os.path.join(GOLDEN, f"driver_{algo}_g500_12_8.log")).read()
    assert p.stdout.startswith("CONFIGURATION:")
    # the reference's configuration keys, in its order, ahead of the GPU's
    cfg_keys = lambda text: [f.split(": ")[0] for f in text.splitlines()[0].split("\t")[1:]]  # noqa: E731
    assert cfg_keys(p.stdout)[:len(cfg_keys(ref))] == cfg_keys(ref)
    assert cfg_keys(p.stdout)[len(cfg_keys(ref)):] == ["DRIVER", "DEVICE", "CUDA_DEVICE", "SM_COUNT", "RUN_NUM"]
    runs = [RUN_LINE.match(x) for x in p.stdout.splitlines() if "th run" in x]
    assert len(runs) == 3 and all(runs)
    assert [int(m.group(1)) for m in runs] == [0, 1, 2]
    for m in runs:
        t = [float(m.group(i)) for i in range(2, 7)]
        assert t[4] == pytest.approx(sum(t[:4]), rel=1e-6, abs=1e-8)
    assert set(verify_triples(p.stdout)) == set(verify_triples(ref))
    assert len(verify_triples(p.stdout)) == 2
    ours, theirs = summary_fields(p.stdout), summary_fields(ref)
    assert [k for k, _ in ours[:len(theirs)]] == [k for k, _ in theirs]
    assert dict(ours)["flop_cnt"] == dict(theirs)["flop_cnt"]
    assert dict(ours)["dataset"] == "g500_12_8" and dict(ours)["num_trials"] == "2"
    assert [k for k, _ in ours[len(theirs):]] == ["gflops", "hbm_frac", "device", "hbm_peak_gbs"]
    # the binary cache written by this run serves the next one with the same result
    assert (ds / "g500_12_8.org.csr").exists() and (ds / "g500_12_8.trs.csr").exists()
    q = subprocess.run([os.path.join(BIN, ALGOS[algo]), "g500_12_8"], cwd=tmp_path, capture_output=True, text=True,
                       env=env, timeout=300)
    assert q.returncode == 0, q.stderr
    assert set(verify_triples(q.stdout)) == set(verify_triples(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["hybacc"])
def test_driver_without_transposed_file(tmp_path, algo):
    """With no <dataset>.trs.mtx, B = A^T is made on the device and the
    driver prints the reference's VERIFYRESULT triple all the same."""
    ds = tmp_path / "dataset"
    subprocess.run([os.path.join(BIN, "cas_gen"), "g500", "12", "8"], check=True, capture_output=True,
                   env=dict(os.environ, CAS_DATASET_DIR=str(ds)))
    (ds / "g500_12_8.trs.mtx").unlink()
    env = dict(os.environ, CAS_RUN_NUM="2", CAS_VERIFY="1")
    p = subprocess.run([os.path.join(BIN, ALGOS[algo]), "g500_12_8"], cwd=tmp_path, capture_output=True, text=True,
                       env=env, timeout=300)
    assert p.returncode == 0, p.stderr
    assert "made on the device" in p.stderr
    ref = open(os.path.join(GOLDEN, f"driver_{algo}_g500_12_8.log")).read()
    assert set(verify_triples(p.stdout)) == set(verify_triples(ref))
    assert dict(summary_fields(p.stdout))["flop_cnt"] == dict(summary_fields(ref))["flop_cnt"]

