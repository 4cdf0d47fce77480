"""bench.py's roofline inputs: every split kernel of every class has a DRAM
traffic figure per face (so the bench line's `traffic` is never null for
the dominant kernel), of the size the ncu captures gave."""
import pytest


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("solver", ["Exact", "HLLC"])
@pytest.mark.parametrize("role", ["gradients", "faces", "update"])
def test_traffic_known_for_every_kernel_of_every_class(dim, solver, role):
    import bench
    t = bench.split_traffic(role, dim, solver, 1_000_000)
    assert t is not None
    assert 40e6 < t < 120e6          # 40-120 bytes per face
    assert bench.split_kernel_name(role, solver).startswith("k_group_s")
