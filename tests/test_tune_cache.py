"""The autotuners' cache file (cola_b200/csrc/tune_cache.h), compiled on the
CPU: a missing file or key misses, an appended line is found again, the first
valid line for a key wins, and lines that do not parse or hold values outside
the launch's search space are skipped -- for the batched tuner's lines and the
single-graph tuner's, which share a file without mixing."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEY = "NVIDIA_B200|148|00112233aabbccdd"


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("tune") / "tune_cache_main")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror",
                           "-I", os.path.join(REPO, "cola_b200", "csrc"),
                           os.path.join(REPO, "tests", "tune_cache_main.cpp"), "-o", out])
    return out


def find(exe, path, key=KEY):
    return subprocess.run([exe, "find", path, key], capture_output=True, text=True, check=True).stdout.split()


def test_missing_file_and_round_trip(exe, tmp_path):
    path = str(tmp_path / "tune.txt")
    assert find(exe, path) == ["miss"]
    subprocess.run([exe, "append", path, KEY, "2", "75", "4", "23.5"], check=True)
    assert find(exe, path) == ["hit", "2", "75", "4", "23.500000"]
    assert find(exe, path, KEY.replace("148", "132")) == ["miss"]  # another SM count is another key


def test_first_valid_line_wins_and_bad_lines_are_skipped(exe, tmp_path):
    path = tmp_path / "tune.txt"
    path.write_text("\n".join([
        "garbage",
        KEY + " 3 100 3 1.0",        # unroll 3 is not a launch option
        KEY + " 4 5 3 1.0",          # grid below 10 %
        KEY + " 4 100 5 1.0",        # 5 blocks per SM is not searched
        KEY + " 4 100",              # truncated
        "other|148|1 2 50 3 2.0",    # another batch
        KEY + " 4 50 3 9.25",        # the first valid line for the key
        KEY + " 2 100 4 1.0",        # a later line for the same key
    ]) + "\n")
    assert find(exe, str(path)) == ["hit", "4", "50", "3", "9.250000"]
    assert find(exe, str(path), "other|148|1") == ["hit", "2", "50", "3", "2.000000"]


def test_append_to_unwritable_path_fails(exe, tmp_path):
    res = subprocess.run([exe, "append", str(tmp_path / "no_dir" / "tune.txt"), KEY, "4", "100", "3", "1"])
    assert res.returncode == 1


SKEY = "spmm|NVIDIA_B200|148|00112233aabbccdd"


def test_single_graph_lines_round_trip_and_validity(exe, tmp_path):
    path = tmp_path / "tune.txt"
    sf = lambda key=SKEY: subprocess.run([exe, "sfind", str(path), key], capture_output=True, text=True,
                                         check=True).stdout.split()
    assert sf() == ["miss"]
    path.write_text("\n".join([
        KEY + " 4 50 3 9.25",               # a batch line: never a single-graph hit
        SKEY + " 96 4 4 0 1.0",             # 96 is not a feature tile
        SKEY + " 128 3 4 0 1.0",            # unroll 3 is not an option
        SKEY + " 128 4 9 0 1.0",            # 9 blocks per SM is not an option
        SKEY + " 128 8 6 0",                # truncated
    ]) + "\n")
    assert sf() == ["miss"]
    subprocess.run([exe, "sappend", str(path), SKEY, "128", "8", "6", "0", "4.5"], check=True)
    subprocess.run([exe, "sappend", str(path), SKEY, "64", "4", "4", "0", "9.0"], check=True)
    assert sf() == ["hit", "128", "8", "6", "0", "4.500000"]
    assert find(exe, str(path)) == ["hit", "4", "50", "3", "9.250000"]  # the batch line still found
