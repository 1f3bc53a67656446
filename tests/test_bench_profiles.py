"""The bench's physical roofline reads DRAM bytes from the committed ncu
summaries (CPU only): every summary the bench names parses to a source hash,
launch options and a byte count, and the traffic is withheld (None, with the
reason) when the built sources or the launch options differ from the
summary's."""
import importlib.util
import os

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("cola_bench", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_committed_profiles_parse():
    bench = load_bench()
    assert bench.PROFILE_FILES
    for workload, name in bench.PROFILE_FILES.items():
        if not os.path.exists(os.path.join(REPO, "profiles", name)):
            continue  # a workload without a capture reports its traffic as null
        prof = bench.read_profile(name)
        assert len(prof.get("build_source_hash", "")) == 16, (workload, prof)
        assert prof.get("launch_options", "").startswith("unroll="), (workload, prof)
        assert int(float(prof["traffic_bytes_per_spmm"])) > 0, (workload, prof)


def test_traffic_withheld_on_other_sources_or_options(monkeypatch):
    bench = load_bench()
    from cola_b200 import _build
    name = bench.PROFILE_FILES["bf16"]
    prof = bench.read_profile(name)
    monkeypatch.setattr(_build, "source_hash", lambda: prof["build_source_hash"])
    traffic, why = bench.profiled_traffic("bf16", prof["launch_options"])
    assert traffic == int(float(prof["traffic_bytes_per_spmm"]))
    assert prof["build_source_hash"] in why
    traffic, why = bench.profiled_traffic("bf16", "unroll=8,min_blocks=0,k_tile=0")
    assert traffic is None and "options" in why
    monkeypatch.setattr(_build, "source_hash", lambda: "0" * 16)
    traffic, why = bench.profiled_traffic("bf16", prof["launch_options"])
    assert traffic is None and "0" * 16 in why
    traffic, why = bench.profiled_traffic("no-such-workload", prof["launch_options"])
    assert traffic is None
