"""The reference-named C++ entry points (include/brig_join_compat.h): a C++ driver, compiled against
the header and linked with libbrigjoin.so the way BRIG-Join's own host code would be, partitions
into the reference's layout, probes, and runs gpu_main over the reference generator's files."""
import json
import os
import subprocess

import numpy as np
import pytest

from gpu_helpers import assert_same_pairs

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
MANIFEST = json.load(open(os.path.join(GOLDEN, "manifest.json")))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("compat") / "compat_driver")
    lib = os.path.join(ROOT, "brig-join_b200", "lib")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(HERE, "compat", "compat_driver.cpp"), "-o", out, "-L", lib, "-lbrigjoin",
                    "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{lib}"], check=True)
    return out


@pytest.mark.parametrize("case", [c for c in MANIFEST if c["R"] > 1], ids=lambda c: c["name"])
@pytest.mark.parametrize("p1,p2", [(16, 5), (512, 67)])
@pytest.mark.parametrize("mode", ["parts", "exec"])
def test_partition_layout_and_probe(driver, oracle, tmp_path, case, p1, p2, mode):
    """parts: partial_jointable_gpu_partition_{r,s}_only then partial_jointable_gpu_run_only_s;
    exec: the same probe through join_execute_host with a one-PE JoinChunkContext."""
    rf, sf = os.path.join(GOLDEN, case["r_file"]), os.path.join(GOLDEN, case["s_file"])
    pairs = str(tmp_path / "pairs.bin")
    r = subprocess.run([driver, mode, rf, sf, str(case["R"]), str(case["S"]), str(p1), str(p2), pairs],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "LAYOUT OK" in r.stdout, r.stdout + r.stderr
    count = int(r.stdout.split("COUNT")[1].split()[0])
    assert count == case["k"]
    raw = np.fromfile(pairs, dtype=np.uint32)
    got_r, got_s = raw[:count], raw[count:]
    rk = np.fromfile(rf, dtype=np.uint32)
    sk = np.fromfile(sf, dtype=np.uint32)
    er, es = oracle.pairs(rk, (np.arange(len(rk)) + 1).astype(np.uint32), sk,
                          (np.arange(len(sk)) + 100000001).astype(np.uint32))
    assert_same_pairs(oracle, got_r, got_s, er, es)


@pytest.mark.parametrize("use_bf", [0, 14])
def test_gpu_main_drop_in(driver, use_bf):
    for case in MANIFEST:
        rf, sf = os.path.join(GOLDEN, case["r_file"]), os.path.join(GOLDEN, case["s_file"])
        r = subprocess.run([driver, "gpu_main", rf, sf, str(case["R"]), str(case["S"]), str(use_bf)],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        assert f"=== Grand Total Answer Count (all PEs): {case['k']} ===" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("case", [c for c in MANIFEST if c["R"] > 1], ids=lambda c: c["name"])
@pytest.mark.parametrize("bits_per_key,k", [(10, 7), (14, 10), (4, 1)])
def test_bloom_filter_object_reference_layout(driver, case, bits_per_key, k):
    """BloomFilter (the reference's object): the filter words built on the device equal a host
    restatement of the reference's placement bit for bit, R's keys all pass, and the S keys that pass
    on the device are those that pass on the host."""
    rf, sf = os.path.join(GOLDEN, case["r_file"]), os.path.join(GOLDEN, case["s_file"])
    bits = bits_per_key * case["R"]
    r = subprocess.run([driver, "bloom", rf, sf, str(case["R"]), str(case["S"]), str(bits), str(k)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "same 1" in r.stdout, r.stdout + r.stderr


REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


@pytest.mark.parametrize("use_bf", [0, 14])
def test_reference_driver_runs_on_the_engine(use_bf):
    """The reference's own command-line driver (src/driver.cpp, unmodified, compiled with its
    CPU check by oracle/Makefile and linked against libbrigjoin.so) joins the golden fixtures on the
    engine: its Grand Total line and its own CPU check both give the known answer."""
    if not os.path.exists(REF_DRIVER):
        pytest.skip("oracle/_ref/ref_driver not built (needs the reference sources at build time)")
    for case in MANIFEST:
        rf, sf = os.path.join(GOLDEN, case["r_file"]), os.path.join(GOLDEN, case["s_file"])
        # rPath sPath outPath R S sanityCheck chunk_size use_bf use_nvlink use_warp_compact true_false_ratio s_chunks
        args = [REF_DRIVER, rf, sf, os.devnull, str(case["R"]), str(case["S"]), "1", "1024", str(use_bf), "0", "0",
                "0.1", "2"]
        r = subprocess.run(args, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        assert f"=== Grand Total Answer Count (all PEs): {case['k']} ===" in r.stdout, r.stdout + r.stderr
        assert f"[sanityCheck] Answer Num (hash-based): {case['k']}" in r.stdout, r.stdout
