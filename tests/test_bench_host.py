"""Host-side pieces of bench.py: the DRAM traffic of the fused kernel comes
from a committed ncu summary (not a literal), the algorithmic bytes follow the
per-particle and per-node figures, and both arms describe the workload with
the same config keys."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_traffic_comes_from_a_committed_profile():
    traffic, source = bench.profile_traffic("c3", "g2p2g")
    assert source is not None and (ROOT / source).is_file()
    assert 1e8 < traffic < 5e8  # one launch on the 128^3 scene moves a few hundred MB
    assert bench.profile_traffic("c3", "no-such-stage") == (None, None)


def test_algorithmic_bytes():
    # 3D: P2G reads x, v, B, F_E, J_p (100 B); G2P reads x, F_E, J_p and writes
    # x, v, B, F_E, J_p (52 + 100 B): 252 B per particle-step
    p2g, g2p = bench.bytes_per_particle(3)
    assert (p2g, g2p, p2g + g2p) == (100, 152, 252)
    p2g2, g2p2 = bench.bytes_per_particle(2)
    assert p2g2 + g2p2 == 132
    grid, gather = bench.bytes_per_node(3)
    assert grid + gather == 112 and gather == 24
    assert sum(bench.bytes_per_node(2)) == 80


def test_config_and_active_nodes():
    """config_of is the one description both arms print; the active-node count
    marks the cubic stencils (int(x) - 1 .. int(x) + 2) inside the grid."""
    import types
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.workload("c1")
    cfg = bench.config_of(types.SimpleNamespace(workload="c1"), sc, 1)
    assert cfg["workload"].startswith("c1: ") and cfg["particles"] == sc.count
    assert set(cfg) == {"workload", "particles", "nodes", "active_nodes_initial", "plasticity", "l2", "parallelism"}
    one = sc.with_(position=sc.position[:1] * 0 + 10.5)  # a single particle in the middle: 4^2 nodes
    assert bench.active_nodes_initial(one) == 16
