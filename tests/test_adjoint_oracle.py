"""The FP64 adjoint oracle (oracle/hvd_adjoint.py) against central finite
differences of the FP64 forward (step 1e-3): the four regulariser scalars
and a random direction in the composite S, through HolographicInit and a
converged 3-outer IRLS refine, on a 24 x 40 crop of an NTSC field. The
lock-in carrier and the anisotropy split are held, as in the adjoint."""
import numpy as np

from hvdg import _cabi, api, synth
from oracle import hvd_adjoint as A
from oracle import hvd_oracle as O

ANISO = 0.8


def _problem():
    g = _cabi.default_geometry(_cabi.STD_NTSC)
    f = synth.make_field(3, _cabi.STD_NTSC, 0.5)
    cfg = api.default_config(irls_outer=3, chroma_aniso=ANISO)
    obs = O.prepare_field(synth.to_ire(f.samples), g, cfg)
    y0, x0, h, w = 100, 200, 24, 40
    sl = (slice(y0, y0 + h), slice(x0, x0 + w))
    return g, cfg, obs.s[sl].copy(), obs.carrier[sl].copy(), f.y_true[sl], f.chi_true[sl]


def _loss(s, c, g, cfg, yt, ct):
    _, _, chi0 = A.init_parts(s, c, g)
    chis = A.refine_forward(s, c, chi0, cfg, ANISO, 1e-14)
    chi = chis[-1]
    y = s - np.real(chi * c)
    return float(np.mean((y - yt) ** 2) + np.mean(np.abs(chi - ct) ** 2)), chis, y, chi


def test_adjoint_matches_central_differences():
    g, cfg, s, c, yt, ct = _problem()
    _, chis, y, chi = _loss(s, c, g, cfg, yt, ct)
    n = y.size
    s_bar, chi0_bar, gl = A.refine_adjoint(s, c, chis, cfg, ANISO, 2 * (y - yt) / n,
                                           2 * (chi - ct) / n, 1e-14)
    s_bar = s_bar + A.init_adjoint(s, c, g, chi0_bar)
    for name, fld in (("lambda_c", "lambda_c"), ("eps", "charbonnier_eps"),
                      ("eps_c", "chroma_eps"), ("k", "structure_coupling")):
        v = getattr(cfg, fld)
        h = 1e-3 * abs(v)
        lp = _loss(s, c, g, _cabi.config_copy(cfg, **{fld: v + h}), yt, ct)[0]
        lm = _loss(s, c, g, _cabi.config_copy(cfg, **{fld: v - h}), yt, ct)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(gl[name] - fd) <= 1e-3 * abs(fd), (name, gl[name], fd)
    rng = np.random.default_rng(0)
    d = rng.normal(size=s.shape)
    h = 1e-3
    fd = (_loss(s + h * d, c, g, cfg, yt, ct)[0] - _loss(s - h * d, c, g, cfg, yt, ct)[0]) / (2 * h)
    an = float(np.sum(s_bar * d))
    assert abs(an - fd) <= 1e-3 * abs(fd), (an, fd)


def test_init_adjoint_is_the_transpose():
    """<J_init dS, v> == <dS, J_init^T v> for the linearised init (FD of the
    forward in a random S direction against the adjoint of a random chi0
    cotangent)."""
    g, cfg, s, c, _, _ = _problem()
    rng = np.random.default_rng(1)
    v = rng.normal(size=s.shape) + 1j * rng.normal(size=s.shape)
    d = rng.normal(size=s.shape)
    h = 1e-4
    jp = (A.init_parts(s + h * d, c, g)[2] - A.init_parts(s - h * d, c, g)[2]) / (2 * h)
    lhs = float(np.sum(np.real(np.conj(v) * jp)))
    rhs = float(np.sum(A.init_adjoint(s, c, g, v) * d))
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), 1e-12), (lhs, rhs)
