"""The bench's byte model and the ncu traffic it reports (CPU only): the
committed summary of the 1M captures holds a traffic line for every kernel
of each workload the bench legs quote, and the standard model counts what
its docstring says."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _bench():
    sys.path.insert(0, str(ROOT))
    import bench
    return bench


def test_traffic_lines_cover_the_quoted_workloads():
    bench = _bench()
    want = {"polydisperse_1m": {"k_topo", "k_contact", "k_force_tiles", "k_walls"},
            "packed_1m": {"k_topo", "k_contact", "k_force_tiles", "k_walls"},
            "tension_254k": {"k_bonds", "k_topo", "k_contact", "k_force_tiles"}}
    for key, kernels in want.items():
        t = bench.profiled_traffic(key)
        assert t is not None, key
        assert set(t["per_kernel"]) == kernels, key
        assert t["bytes_per_step"] == sum(t["per_kernel"].values())
        assert all(v > 0 for v in t["per_kernel"].values())
    assert bench.profiled_traffic("no_such_workload") is None


def test_standard_byte_model():
    bench = _bench()
    step, whole, tight = bench.algorithmic_bytes(1_000_000, 250_000, 6_000_000, 1000)
    assert step == 368 * 1_000_000 + 52 * 6_000_000
    assert whole == step + 16 * 1_000_000 + 16 * 250_000 + 136 * 1000
    assert tight <= step
