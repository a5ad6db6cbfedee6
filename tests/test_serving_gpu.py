"""Solve server (continuous batching): uneven requests (cells, k-points,
band counts) admitted by device footprint and solved concurrently, each on
its own stream.

Checks: a request's eigenvalues and residuals are bit-identical whether it is
served alone (one slot) or in the mix (three slots, overlapping solves), and
within 1e-10 Ha of the reference's solve where a fixture exists; the
admission never budgets above the memory cap (a cap that fits one solve runs
them one at a time); a request that cannot fit is refused at submit."""
import numpy as np
import pytest

from sdft_b200 import _capi as C
from sdft_b200 import synthetic
from sdft_b200.serving import SolveServer, solve_footprint

pytestmark = pytest.mark.gpu


def _requests():
    return [
        ("tiny", synthetic.tiny(), "fp64"),
        ("gaas_k26", synthetic.gaas_small((1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0)), "mixed"),
        ("tiny_k", synthetic.tiny(seed=9, kpoint=(0.5, 0.0, 0.25), roots=5), "mixed"),
        ("gaas_k13", synthetic.gaas_small((0.0, 1.0 / 3.0, 1.0 / 3.0)), "fp64"),
        ("si8", synthetic.si8(), "mixed"),
        ("tiny_b", synthetic.tiny(seed=11, ecut_ha=5.0, roots=9), "fp64"),
    ]


def _serve(requests, slots, cap=64e9):
    with SolveServer(0, cap, slots) as server:
        tickets = [server.submit(x, precision=p) for _, x, p in requests]
        results = [server.wait(t) for t in tickets]
        memory = server.memory()
    return results, memory


@pytest.fixture(scope="module")
def served(context):
    requests = _requests()
    alone, _ = _serve(requests, 1)
    mixed, memory = _serve(requests, 3)
    return requests, alone, mixed, memory


def test_results_identical_alone_and_in_the_mix(served):
    requests, alone, mixed, _ = served
    for (name, _, _), a, m in zip(requests, alone, mixed):
        assert a["converged"] and m["converged"], name
        assert np.array_equal(a["eigenvalues"], m["eigenvalues"]), name
        assert np.array_equal(a["residuals"], m["residuals"]), name
        assert np.max(m["residuals"]) <= 1e-12, name


def test_results_match_reference_fixtures(served, golden):
    requests, _, mixed, _ = served
    for (name, _, _), m in zip(requests, mixed):
        if name in ("tiny", "si8", "gaas_k13", "gaas_k26"):
            assert np.max(np.abs(m["eigenvalues"] - golden(name)["eigenvalues"])) < 1e-10, name


def test_solves_overlap_in_the_mix(served):
    _, alone, mixed, memory = served
    spans = sorted((r["timing"]["started"], r["timing"]["finished"]) for r in mixed)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    assert len({r["timing"]["slot"] for r in mixed}) > 1
    one = sorted((r["timing"]["started"], r["timing"]["finished"]) for r in alone)
    assert all(one[i + 1][0] >= one[i][1] for i in range(len(one) - 1))
    assert memory["in_use"] == 0 and 0 < memory["peak"] <= memory["cap"]


def test_admission_respects_the_memory_cap(context):
    requests = _requests()[:3]
    largest = max(solve_footprint(x, x.roots) for _, x, _ in requests)
    results, memory = _serve(requests, 3, cap=1.5 * largest)
    assert all(r["converged"] for r in results)
    assert memory["peak"] <= memory["cap"]
    # Solves that ran at the same time fit under the cap together.
    for i, a in enumerate(results):
        for b in results[i + 1:]:
            ta, tb = a["timing"], b["timing"]
            if ta["started"] < tb["finished"] and tb["started"] < ta["finished"]:
                assert ta["footprint"] + tb["footprint"] <= memory["cap"]


def test_request_above_the_cap_is_refused(context):
    x = synthetic.tiny()
    with SolveServer(0, solve_footprint(x, x.roots) // 2, 1) as server:
        with pytest.raises(C.InvalidArgument, match="exceeds the server memory cap"):
            server.submit(x)


def test_unknown_ticket_is_refused(context):
    with SolveServer(0, 1e9, 1) as server:
        with pytest.raises(C.InvalidArgument, match="unknown solve ticket"):
            server.wait(12345, timeout=0.0)
