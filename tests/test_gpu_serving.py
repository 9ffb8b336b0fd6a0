"""Batched and served proving: every proof made concurrently with others is
the same bytes as the plain single-proof call, admission respects the HBM
budget, and the request API reports timeouts and bad configs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _alone(lg, ctx, sizes, seeds):
    out = []
    for L, s in zip(sizes, seeds):
        cfg = lg.config_for_size(L)
        out.append(lg.prover(cfg, lg.splitmix_coeffs_device(s, cfg.poly_len, ctx), ctx).to_bytes())
    return out


def test_prove_batch_uneven_sizes_match_single_proofs(lg, ctx):
    rng = np.random.default_rng(3)
    sizes = [int(x) for x in rng.integers(16, 21, size=12)]
    seeds = [3 * 2**32 + i for i in range(12)]
    want = _alone(lg, ctx, sizes, seeds)
    cfgs = [lg.config_for_size(L) for L in sizes]
    polys = [lg.splitmix_coeffs_device(s, c.poly_len, ctx) for s, c in zip(seeds, cfgs)]
    got = [p.to_bytes() for p in lg.prove_batch(cfgs, polys, workers=4)]
    assert got == want


def test_server_mixed_stream_with_budget(lg, ctx):
    # budget for about two 2^20 proofs at a time; 16 requests of mixed size
    sizes = [16, 20, 17, 18, 20, 16, 19, 16, 20, 18, 17, 16, 19, 20, 16, 18]
    seeds = [4 + i for i in range(len(sizes))]
    want = _alone(lg, ctx, sizes, seeds)
    # admission charges the contexts' own arenas and tables as well
    cached = 4 * lg.lib.lg_ctx_device_bytes_cached(ctx.handle) + (64 << 20)
    srv = lg.Server(0, workers=4, hbm_budget_bytes=cached + 2 * (28 << 20) + 2 * (48 << 20))
    try:
        tickets = []
        for L, s in zip(sizes, seeds):
            cfg = lg.config_for_size(L)
            tickets.append(srv.submit(cfg, lg.splitmix_coeffs(s, cfg.poly_len), copy_input=True))
        got = []
        for t in tickets:
            proof, lat, queue = srv.wait(t)
            assert lat >= queue >= 0
            got.append(proof.to_bytes())
        assert got == want
        st = srv.stats()
        assert st["completed"] == len(sizes) and st["queued"] == 0 and st["in_flight_bytes"] == 0
    finally:
        srv.close()


def test_server_device_inputs_timeout_and_errors(lg, ctx):
    srv = lg.Server(0, workers=2)
    try:
        cfg = lg.hardcoded_config_24()
        poly = lg.splitmix_coeffs_device(1, cfg.poly_len, ctx)
        t = srv.submit(cfg, poly)
        first = srv.wait(t, timeout_ms=0)  # most likely still running
        if first is None:
            proof, lat, _ = srv.wait(t)
        else:
            proof, lat, _ = first
        assert lat > 0
        assert proof.to_bytes() == lg.prover(cfg, poly, ctx).to_bytes()
        with pytest.raises(lg.LigeritoError) as e:
            srv.submit(cfg, lg.splitmix_coeffs(0, 1 << 16))  # wrong length for config 24
        assert e.value.status == 2
    finally:
        srv.close()


def test_single_worker_server_is_fifo(lg, ctx):
    srv = lg.Server(0, workers=1)
    try:
        cfgs = [lg.config_for_size(L) for L in (18, 16, 17)]
        tickets = [srv.submit(c, lg.splitmix_coeffs(i, c.poly_len), copy_input=True) for i, c in enumerate(cfgs)]
        results = [srv.wait(t) for t in tickets]
        # with one worker each request waits for everything submitted before it
        lats = [r[1] for r in results]
        assert lats[0] <= lats[1] <= lats[2]
    finally:
        srv.close()


def test_two_waiters_on_one_ticket_get_one_result(lg, ctx):
    # the result is handed out once; the other waiter is told the ticket is
    # gone instead of reading a freed request
    import threading

    srv = lg.Server(0, workers=1)
    try:
        cfg = lg.config_for_size(20)
        t = srv.submit(cfg, lg.splitmix_coeffs_device(20, cfg.poly_len, ctx))
        out = []

        def waiter():
            try:
                out.append(("proof", srv.wait(t)[0].to_bytes()))
            except lg.LigeritoError as e:
                out.append(("error", e.status))

        ths = [threading.Thread(target=waiter) for _ in range(3)]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        assert sorted(k for k, _ in out) == ["error", "error", "proof"]
        assert all(v == 1 for k, v in out if k == "error")
        with pytest.raises(lg.LigeritoError) as e:
            srv.wait(t)
        assert e.value.status == 1
    finally:
        srv.close()


def test_server_warm_then_same_bytes(lg, ctx):
    srv = lg.Server(0, workers=3)
    try:
        cfgs = [lg.config_for_size(L) for L in (16, 18)]
        srv.warm(cfgs)
        assert srv.stats()["completed"] == 6
        want = _alone(lg, ctx, [18], [77])[0]
        t = srv.submit(cfgs[1], lg.splitmix_coeffs_device(77, cfgs[1].poly_len, ctx))
        assert srv.wait(t)[0].to_bytes() == want
    finally:
        srv.close()


@pytest.mark.parametrize("host_input", [False, True])
def test_server_lockstep_batches_match_single_proofs(lg, ctx, host_input):
    # max_batch 8: queued requests of one size are proved in lockstep
    # groups; every proof is still the single-proof bytes
    sizes = [16, 16, 17, 16, 18, 17, 16, 16, 17, 18, 16, 17, 16, 16, 18, 16, 17, 16, 16, 16]
    seeds = [900 + i for i in range(len(sizes))]
    want = _alone(lg, ctx, sizes, seeds)
    srv = lg.Server(0, workers=2, max_batch=8)
    try:
        tickets = []
        for L, s in zip(sizes, seeds):
            cfg = lg.config_for_size(L)
            poly = lg.splitmix_coeffs(s, cfg.poly_len) if host_input else lg.splitmix_coeffs_device(s, cfg.poly_len, ctx)
            tickets.append(srv.submit(cfg, poly, copy_input=host_input))
        got = [srv.wait(t)[0].to_bytes() for t in tickets]
        assert got == want
        st = srv.stats()
        assert st["completed"] == len(sizes) and st["in_flight_bytes"] == 0
    finally:
        srv.close()
    with pytest.raises(lg.LigeritoError):
        lg.Server(0, workers=1, max_batch=65)
