"""The serving loop: mixed requests (B, N, alpha, analysis/synthesis) arriving
while others run give exactly the results they give alone, and the latency
statistics are well formed."""
import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("use_graphs,priorities", [(True, False), (False, False), (True, True)])
def test_results_identical_alone_and_in_mix(use_graphs, priorities):
    from s2dw_b200.serving import Server, make_stream

    reqs, inputs = make_stream(40, seed=3, rate_hz=20000.0, Bs=(32, 48, 64, 128, 256, 512), Ns=range(1, 9),
                               alphas=(2.0, 3.0), pool=2)
    # in the mix: everything arrives within ~2 ms, many requests overlap
    # (with priorities, the small requests' kernels overtake the larger ones')
    srv = Server(hbm_budget_bytes=8 << 30, slots_per_config=2, use_graphs=use_graphs, keep_outputs=True,
                 priorities=priorities)
    stats = srv.run(reqs)
    srv.close()
    assert stats["requests"] == len(reqs)
    assert 0 < stats["p50_ms"] <= stats["p99_ms"]
    mixed = {r.rid: r.out for r in reqs}
    # alone: one request at a time, fresh server
    alone_srv = Server(hbm_budget_bytes=8 << 30, slots_per_config=1, use_graphs=False, keep_outputs=True)
    for r in reqs:
        r.arrival = 0.0
        r.out = None
        alone_srv.run([r])
        for a, b in zip(r.out, mixed[r.rid]):
            np.testing.assert_array_equal(a, b)
    alone_srv.close()


@pytest.mark.gpu
def test_synthesis_requests_reconstruct_their_maps():
    from s2dw_b200.serving import Server, make_stream

    reqs, inputs = make_stream(24, seed=5, rate_hz=5000.0, Bs=(64, 96), Ns=(2, 5), alphas=(2.0,), pool=2)
    srv = Server(hbm_budget_bytes=4 << 30, keep_outputs=True)
    srv.run(reqs)
    srv.close()
    for r in reqs:
        if r.kind != "synthesis":
            continue
        lst = inputs[(r.B, r.N, r.alpha, r.J)]
        flm_ref = next(f for (_, w, _, f) in lst if w.data_ptr() == r.inp[0].data_ptr())
        f = r.out[0].T
        assert np.abs(f - flm_ref).max() < 1e-12


@pytest.mark.gpu
def test_budget_evicts_idle_slots():
    from s2dw_b200.serving import Server, Slot, make_stream

    reqs, _ = make_stream(30, seed=7, rate_hz=50000.0, Bs=(64, 128), Ns=(1, 3, 4, 7), alphas=(2.0, 3.0), pool=1)
    small = Slot.estimate_bytes(128, 7, 2.0, 7) * 3  # room for about three slots
    srv = Server(hbm_budget_bytes=small, slots_per_config=1)
    stats = srv.run(reqs)
    assert stats["requests"] == len(reqs)
    assert srv.used <= small
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("use_graphs", [True, False])
def test_split_form_batches_and_results_identical_alone(use_graphs):
    """Split-form serving: waiting requests of one configuration and kind run
    as one tensor-core batch; each result equals the result of the same
    request served alone (a batch of one), bit for bit, and the FP64 form's
    within the split form's tolerance (1e-10 relative to the largest output)."""
    from s2dw_b200.serving import Server, make_stream

    reqs, inputs = make_stream(48, seed=11, rate_hz=50000.0, Bs=(32, 64, 128), Ns=(2, 5), alphas=(2.0,), pool=2)
    srv = Server(hbm_budget_bytes=16 << 30, slots_per_config=1, use_graphs=use_graphs, keep_outputs=True,
                 form="split")
    stats = srv.run(reqs)
    srv.close()
    assert stats["requests"] == len(reqs)
    assert stats["form"] == "split"
    assert stats["mean_batch"] > 1.0
    assert 0 < stats["p50_ms"] <= stats["p99_ms"]
    mixed = {r.rid: r.out for r in reqs}

    alone_srv = Server(hbm_budget_bytes=16 << 30, slots_per_config=1, use_graphs=False, keep_outputs=True,
                       form="split")
    fp64_srv = Server(hbm_budget_bytes=16 << 30, slots_per_config=1, use_graphs=False, keep_outputs=True)
    for r in reqs:
        r.arrival = 0.0
        r.out = None
        alone_srv.run([r])
        for a, b in zip(r.out, mixed[r.rid]):
            np.testing.assert_array_equal(a, b)
        r.out = None
        fp64_srv.run([r])
        for a, b in zip(r.out, mixed[r.rid]):
            assert np.abs(a - b).max() <= 1e-10 * np.abs(a).max()
    alone_srv.close()
    fp64_srv.close()
