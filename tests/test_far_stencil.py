"""Host side of the mixed path's far wake term: the evaluation points and stencils that
far_wake_stencil builds for smooth patches of the ring grid (no GPU)."""
import numpy as np
import pytest

from pyvl_b200.engine import column_stencil, far_wake_stencil


def _apply(plan, values):
    """Numpy restatement of pvl_stencil_normal_add without the normal: (n_rings, 3)."""
    off, ent, w = plan["offsets"].astype(np.int64), plan["entries"].astype(np.int64), plan["weights"]
    out = np.zeros((off.size - 1, values.shape[1]))
    for p in range(off.size - 1):
        k = slice(off[p], off[p + 1])
        out[p] = (w[k, None] * values[ent[k]]).sum(0)
    return out


def _field(i, j):
    """Products of quintics in the two grid directions: what the quintic midpoint rules reproduce."""
    return np.stack([(0.3 + 0.1 * i - 0.002 * i ** 3 + 1e-6 * i ** 5) * (1.0 - 0.05 * j + 0.01 * j ** 2),
                     np.cos(0.0) + 0.0 * i + 1e-4 * j ** 5,
                     1e-7 * i ** 5 * j ** 4 - 0.2 * j], axis=1)


@pytest.mark.parametrize("patches", [((0, 64, 32), (2048, 64, 32)), ((0, 128, 32),), ((5, 20, 11), (300, 7, 13))])
def test_stencil_reproduces_quintics(patches):
    n = 4096
    plan = far_wake_stencil(n, patches)
    idx = plan["index"].astype(np.int64)
    n_c, n_s = plan["n_chord_eval"], plan["n_span_eval"]
    assert idx.size == n_c and np.unique(idx).size == n_c and n_s <= n_c
    # grid coordinates of every ring (rings outside the patches: a field that is not smooth at all)
    ii = np.zeros(n)
    jj = np.zeros(n)
    rng = np.random.default_rng(0)
    inside = np.zeros(n, bool)
    for r0, ns, nc in patches:
        k = np.arange(ns * nc)
        ii[r0 + k], jj[r0 + k] = k // nc, k % nc
        inside[r0 + k] = True
    f = _field(ii, jj)
    f[~inside] = rng.normal(size=(int((~inside).sum()), 3))
    chord_only = np.zeros((n_c + n_s, 3))
    chord_only[:n_c] = f[idx]
    np.testing.assert_allclose(_apply(plan, chord_only), f, rtol=0, atol=1e-12 * np.abs(f).max())
    span_only = np.zeros((n_c + n_s, 3))
    span_only[n_c:] = f[idx[:n_s]]
    np.testing.assert_allclose(_apply(plan, span_only), f, rtol=0, atol=1e-12 * np.abs(f).max())
    # rings outside every patch are evaluated in both bands and take their own values
    out = np.nonzero(~inside)[0]
    assert np.isin(out, idx[:n_s]).all()


def test_stencil_counts_of_the_flapping_halves():
    """128 x 32 rings as two 64 x 32 halves: 21 of 32 chordwise points evaluated (the even ones
    and the five within reach of an edge), 37 of 64 spanwise per half."""
    plan = far_wake_stencil(4096, ((0, 64, 32), (2048, 64, 32)))
    assert plan["n_chord_eval"] == 128 * 21
    assert plan["n_span_eval"] == 2 * 37 * 21
    # 1 + 36 terms at most: a point's chord band rule has 1 or 6, its span band rule up to 6 x 6
    assert np.diff(plan["offsets"].astype(np.int64)).max() == 6 + 36


def test_stencil_rejects_bad_patches():
    with pytest.raises(ValueError):
        far_wake_stencil(100, ((0, 10, 11),))
    with pytest.raises(ValueError):
        far_wake_stencil(100, ((0, 5, 10), (40, 2, 10)))
    with pytest.raises(ValueError):
        far_wake_stencil(100, ((-1, 2, 2),))
    plan = far_wake_stencil(100, ())
    assert plan["n_chord_eval"] == plan["n_span_eval"] == 100
    assert (plan["weights"] == 1.0).all()


def test_column_stencil_reproduces_quintics():
    """129 trailing-edge node columns as two runs sharing the root column 64: 73 evaluated (the
    even ones and those within five of a run end), every column of a quintic field exact."""
    plan = column_stencil(129, ((0, 65), (64, 65)))
    sub = plan["sub"]
    assert sub.size == 73 and 64 in sub and 0 in sub and 128 in sub
    c = np.arange(129, dtype=np.float64)
    x = np.where(c <= 64, c, 128.0 - c)  # a kink at the shared column: each run smooth on its own
    f = np.stack([1 + 0.01 * x - 1e-4 * x ** 3 + 1e-8 * x ** 5, np.ones(129), x ** 2], axis=1)
    off, ent, w = plan["offsets"].astype(np.int64), plan["entries"].astype(np.int64), plan["weights"]
    got = np.array([(w[off[k]:off[k + 1], None] * f[sub][ent[off[k]:off[k + 1]]]).sum(0) for k in range(129)])
    np.testing.assert_allclose(got, f, rtol=0, atol=1e-9 * np.abs(f).max())


def test_column_stencil_rejects_bad_runs():
    with pytest.raises(ValueError):
        column_stencil(20, ((0, 21),))
    with pytest.raises(ValueError):  # column 15 inside both runs
        column_stencil(40, ((0, 30), (10, 30)))
    plan = column_stencil(12, ())
    assert plan["sub"].size == 12 and (plan["weights"] == 1.0).all()
