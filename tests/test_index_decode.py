"""The grid index decoding of the CUDA library (common.cuh: div_r, cell_ijk, face_ijk) for every
supported grid size.

The kernels find a cell's or a face's (i, j, k) without integer division: q = trunc(x * r) with r
the double reciprocal of the divisor (computed on the host, make_scene in host.cu), then one
correction by the remainder.  Every step is an IEEE double operation (a correctly rounded
reciprocal, a correctly rounded product, truncation), which numpy performs with the same bits,
so this checks the arithmetic itself at the values where it could fail: the multiples of each
divisor and their neighbours, for n = 2 .. 1024 (the sizes scenes are validated to), up to the
largest face index of the largest scene.  The GPU parity tests check the kernels that use it.
"""
import numpy as np


def _div_r(x, d, r):
    q = (x.astype(np.float64) * r).astype(np.int64)  # truncation toward zero, as (long long)
    rem = x - q * d
    return q + np.where(rem < 0, -1, np.where(rem >= d, 1, 0))


def test_div_r_exact_for_every_grid_size():
    rng = np.random.default_rng(3)
    for n in range(2, 1025):
        dn = float(n)
        per = n * n * (n + 1)
        top = 3 * per  # faces of one scene: the largest local index decoded
        for d, r in ((n, 1.0 / dn), (n + 1, 1.0 / (dn + 1.0)), (n * n, 1.0 / (dn * dn)),
                     (n * (n + 1), 1.0 / (dn * (dn + 1.0)))):
            qmax = top // d + 1
            q = np.unique(np.concatenate([np.arange(min(qmax, 64)), rng.integers(0, qmax, 256),
                                          np.arange(max(qmax - 64, 0), qmax)]))
            x = (q[:, None] * d + np.array([-1, 0, 1, d - 1])[None, :]).ravel()
            x = x[(x >= 0) & (x <= top)]
            got = _div_r(x, d, r)
            assert np.array_equal(got, x // d), (n, d)


def test_face_decode_round_trip_small_grids():
    """face_ijk's plane and row divisors per axis, restated, invert the face layout of every
    face of grids up to 24^3."""
    for n in (2, 3, 5, 7, 16, 24):
        dn = float(n)
        inv = {n: 1.0 / dn, n + 1: 1.0 / (dn + 1.0), n * n: 1.0 / (dn * dn), n * (n + 1): 1.0 / (dn * (dn + 1.0))}
        per = n * n * (n + 1)
        f = np.arange(3 * per, dtype=np.int64)
        axis = (f >= per).astype(np.int64) + (f >= 2 * per)
        r = f - axis * per
        rowd = np.where(axis == 0, n * n, (n + 1) * n)
        kd = np.where(axis == 2, n + 1, n)
        a = np.empty_like(r)
        b = np.empty_like(r)
        for ax in range(3):
            m = axis == ax
            rd, kk = int(rowd[m][0]), int(kd[m][0])
            a[m] = _div_r(r[m], rd, inv[rd])
            b[m] = _div_r(r[m] - a[m] * rd, kk, inv[kk])
        k = r - a * rowd - b * kd
        # the layouts: x faces (i n + j) n + k, y faces (i (n+1) + j) n + k, z faces (i n + j)(n+1) + k
        ej = np.where(axis == 1, n + 1, n)
        ek = np.where(axis == 2, n + 1, n)
        assert np.array_equal((a * ej + b) * ek + k, r)
        assert (k >= 0).all() and (k < ek).all() and (b >= 0).all() and (b < ej).all()
