"""Host-side pieces of bench.py that need no GPU: the roofline's DRAM traffic
read from the committed ncu summaries, the algorithmic-byte tables, and the error
report's per-field arithmetic."""
import numpy as np

import bench


def test_profile_traffic_reads_the_committed_summaries():
    """The bench line's roofline.traffic comes from profiles/<kernel>_<workload>_<precision>.txt."""
    for k in ("k_move_fused", "k_cellnodes"):
        t = bench.profile_traffic(k)
        assert t is not None and 0.0 < t < 200.0, k
    assert bench.profile_traffic("k_no_such_kernel") is None


def test_algorithmic_byte_tables_add_up():
    """Per marker 33 B read + 24 B written, per node 24 B read + 64 B written; the
    general path's per-phase shares add up to those totals, and the fused path's
    dominant kernel carries every marker byte."""
    assert bench.B_MARKER == 57 and bench.B_NODE == 88
    assert sum(v[1] for v in bench.KERNEL_BYTES.values()) == bench.B_MARKER
    assert sum(v[2] for v in bench.KERNEL_BYTES.values()) == bench.B_NODE
    assert bench.FUSED_KERNEL_BYTES["movemark"][1] == bench.B_MARKER
    assert sum(v[2] for v in bench.FUSED_KERNEL_BYTES.values()) == bench.B_NODE


def test_field_errors():
    ref = {"a": np.array([1.0, -2.0, 4.0]), "b": np.zeros(3)}
    got = {"a": np.array([1.0, -2.0, 4.0 + 4e-7]), "b": np.zeros(3)}
    e = bench.field_errors(got, ref, ("a", "b"))
    assert abs(e["a"]["max_rel"] - 1e-7) < 1e-12
    assert abs(e["a"]["l2_rel"] - 4e-7 / np.sqrt(21.0)) < 1e-12
    assert e["b"] == {"max_rel": 0.0, "l2_rel": 0.0}
