"""The bench's measurement model on CPU: the algorithmic bytes per kernel
follow the per-unit figures (ray segment 80 B + 32 B per node + 52 B per
surfel test; lookup 36 B per photon + 8 B per window row; the adjoint
bounce's pending state and inter-kernel records; 72 B per gradient event),
every timed kernel group has a DRAM traffic entry for the roofline, and
the counters the bench line reports are the ones the model reads."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import bench  # noqa: E402


def _counters():
    sf = {k: 0 for k in bench.FWD_COUNTERS}
    sb = {k: 0 for k in bench.ADJ_COUNTERS}
    sf.update(gather_segments=1000, gather_node_visits=30000, gather_surfel_tests=5000, gather_queries=900,
              gather_photons_scanned=45000)
    sb.update(adjoint_segments=700, node_visits=20000, surfel_tests=3000, gradient_events=300, gather_queries=200,
              photons_scanned=7000)
    return sf, sb


def test_algorithmic_bytes_follow_the_unit_figures():
    sf, sb = _counters()
    kb = bench.kernel_bytes(sf, sb)
    rows = bench.ROWS_PER_QUERY
    assert kb["k_cg_round"] == 80 * 1000 + 32 * 30000 + 52 * 5000
    assert kb["k_cg_lookup"] == 36 * 45000 + 8 * rows * 900
    assert kb["k_adj_bounce"] == 80 * 700 + 32 * 20000 + 52 * 3000 + (96 + 128) * 700
    assert kb["k_transport"] == 72 * 300 + 36 * 7000 + 8 * rows * 200


def test_every_timed_kernel_has_traffic_and_counters():
    sf, sb = _counters()
    timed = set(bench.kernel_bytes(sf, sb))
    with open(os.path.join(os.path.dirname(HERE), "profiles", "traffic.json")) as f:
        traffic = json.load(f)
    assert timed <= set(traffic), timed - set(traffic)
    rates = {k: v["dram_bytes_per_s"] for k, v in traffic.items() if not k.startswith("_")}
    assert all(isinstance(v, int) and v > 0 for v in rates.values())
    for k in timed:
        # the DRAM rate of the small-case capture times the launch's time
        assert bench.read_traffic(k, 2.0) == int(rates[k] * 2.0 / 1e3)
    gather = set(bench.kernel_bytes(sf, dict(sb, vertex_entries=10, vertex_records=40), "gather"))
    assert gather <= set(rates), gather - set(rates)
    # the model reads only counters the bench line reports
    assert {"gather_segments", "gather_node_visits", "gather_surfel_tests", "gather_queries",
            "gather_photons_scanned"} <= set(bench.FWD_COUNTERS)
    assert {"adjoint_segments", "node_visits", "surfel_tests", "gradient_events", "gather_queries",
            "photons_scanned"} <= set(bench.ADJ_COUNTERS)
