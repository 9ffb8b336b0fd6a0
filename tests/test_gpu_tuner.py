"""The autotuner changes speed only: with it on, transforms and proofs are
the same bytes as with the default stage split and fold grid, and the
choices it made are listed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotuned_proofs_and_ffts_match(lg, ref, ctx):
    cfg = lg.config_for_size(18)
    poly = lg.splitmix_coeffs_device(18, cfg.poly_len, ctx)
    want = lg.prover(cfg, poly, ctx).to_bytes()
    tuned = lg.Context(0)
    try:
        tuned.set_autotune(True)
        assert lg.prover(cfg, poly, tuned).to_bytes() == want
        assert lg.prover(cfg, poly, tuned).to_bytes() == want  # with the tuned choices cached
        v = lg.splitmix_coeffs(31, 3 << 14)
        d = lg.to_device(v)
        lg.fft(d, 14, tuned)
        tw = ref.twiddles(14)
        got = lg.to_host(d).reshape(3, -1)
        for i in range(3):
            assert (got[i] == ref.fft(v.reshape(3, -1)[i], tw=tw)).all()
    finally:
        tuned.close()
    choices = lg.tuned_choices()
    assert any(c.startswith("fft ") for c in choices)
    assert any(c.startswith("fold ") for c in choices)
