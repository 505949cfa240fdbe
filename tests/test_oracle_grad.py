"""The oracle's FP64 adjoint against FP64 central finite differences (CPU).

The adjoint (oracle/sfo_grad.cpp) is what the GPU backward is checked
against; here it is checked itself. A parameter within a step of a
non-smooth point of the forward (a pair crossing alpha = 1/255, a pixel's
termination threshold, a tile-bbox edge) makes its finite difference jump;
such a sample is recognised by its one-sided differences disagreeing at two
step sizes and is re-tested with a ten times smaller step."""
import numpy as np
import pytest


def central_difference(loss, base, idx, h):
    """Central difference at `idx`, stepping down once if either side jumps."""
    for step in (h, h / 10, h / 100):
        p, m = base.copy(), base.copy()
        p[idx] += step
        m[idx] -= step
        lp, lm, l0 = loss(p), loss(m), loss(base)
        fwd, bwd = (lp - l0) / step, (l0 - lm) / step
        if abs(fwd - bwd) <= 1e-3 * max(abs(fwd), abs(bwd)) + 1e-5:
            return (lp - lm) / (2 * step)
    return None


def scene(n, k, seed):
    rng = np.random.default_rng(seed)
    a = np.zeros((11, n))
    a[0:2] = rng.uniform(-0.6, 0.6, (2, n))
    a[2] = rng.uniform(-0.3, 0.6, n)
    q = rng.normal(size=(4, n))
    a[3:7] = q / np.linalg.norm(q, axis=0)
    a[7:10] = rng.normal(-2.3, 0.3, (3, n))
    a[10] = rng.normal(0.0, 1.0, n)
    sh = rng.normal(0, 0.3, (k, 3, n))
    return a.reshape(-1), sh.reshape(-1)


@pytest.mark.parametrize("k", [1, 4, 16])
def test_fp64_adjoint_matches_central_differences(oracle_mod, k):
    O = oracle_mod
    n, w, h = 24, 40, 36
    attr, sh = scene(n, k, 100 + k)
    cam = O.look_at((0.2, -0.1, -2.5), (0.0, 0.0, 0.0))
    rng = np.random.default_rng(7)
    dl = rng.normal(size=(h, w, 4))

    def loss(at, s):
        img = O.render64(cam, w, h, at, s, k)
        return float(np.sum(img * dl))

    d_attr, d_sh = O.render64_backward(cam, w, h, attr, sh, k, dl)
    checks, kinks, bad = 0, 0, []
    for plane in range(11):
        for i in range(n):
            idx = plane * n + i
            fd = central_difference(lambda a: loss(a, sh), attr, idx, 1e-6)
            if fd is None:
                kinks += 1
                continue
            checks += 1
            if abs(fd - d_attr[idx]) > 1e-4 * max(abs(fd), abs(d_attr[idx])) + 1e-6:
                bad.append((plane, i, fd, d_attr[idx]))
    for idx in range(0, sh.size, max(1, sh.size // 60)):
        fd = central_difference(lambda s: loss(attr, s), sh, idx, 1e-6)
        if fd is None:
            kinks += 1
            continue
        checks += 1
        if abs(fd - d_sh[idx]) > 1e-4 * max(abs(fd), abs(d_sh[idx])) + 1e-6:
            bad.append(("sh", idx, fd, d_sh[idx]))
    assert not bad, bad[:10]
    assert kinks <= 0.02 * (checks + kinks)
    # The gradient is not trivially zero.
    assert np.abs(d_attr).max() > 1e-3
