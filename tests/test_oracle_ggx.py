"""The oracle's GGX rough-metal sampler (the library's GGX_METAL extension;
Walter, Marschner, Li and Torrance, EGSR 2007) checked against properties of
the published model, in FP64 on the CPU:
  * directions are unit vectors on the lit side of the surface;
  * the half vectors m = normalize(i + o) follow the GGX distribution of
    D(m)|m.n|, whose CDF in theta_m is tan^2 / (alpha^2 + tan^2) (eq. 35);
  * with F0 = 1 the mean sample weight is the single-scattering directional
    albedo: at most 1 (energy conservation), near 1 for a nearly smooth
    surface, and lower for a rough one at grazing incidence;
  * as alpha -> 0 the reflection tends to the mirror direction."""
import numpy as np
import pytest

import _oracle as O

N = np.array([0.0, 0.0, 1.0])


def incoming(theta):
    # d points towards the surface; i = -d makes angle theta with n.
    return np.array([-np.sin(theta), 0.0, -np.cos(theta)])


@pytest.mark.parametrize("alpha", [0.05, 0.3, 0.6])
@pytest.mark.parametrize("theta", [0.0, 0.7, 1.3])
def test_directions_and_energy(alpha, theta):
    n = 200000
    d, w, ok = O.ggx_samples(incoming(theta), N, np.ones(3), alpha, 1, n)
    assert ok.mean() > 0.5
    dd = d[ok]
    assert np.allclose(np.linalg.norm(dd, axis=1), 1.0, atol=1e-12)
    assert (dd[:, 2] > 0).all()
    assert np.isfinite(w).all() and (w >= 0).all()
    # Weights of the paths that end count as zero.
    e = w[:, 0]
    mean, se = e.mean(), e.std() / np.sqrt(n)
    assert mean <= 1.0 + 4 * se, (mean, se)
    if alpha == 0.05 and theta < 1.0:
        assert mean > 0.985
    if alpha == 0.6 and theta > 1.2:
        assert mean < 0.95  # single scattering loses energy at grazing angles


@pytest.mark.parametrize("alpha", [0.1, 0.4])
def test_half_vectors_follow_ggx(alpha):
    n = 100000
    i = -incoming(0.3)
    d, _, ok = O.ggx_samples(incoming(0.3), N, np.ones(3), alpha, 7, n)
    m = d[ok] + i
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    c = np.clip(m[:, 2], 0.0, 1.0)
    t2 = (1.0 - c * c) / (c * c)
    u = t2 / (alpha * alpha + t2)
    # Kolmogorov-Smirnov distance of u against uniform.  Paths that end drop
    # the m with i.m <= 0 or o below the surface, a small biased fraction at
    # this incidence; the bound allows for it.
    u = np.sort(u)
    ks = np.max(np.abs(u - (np.arange(1, len(u) + 1) - 0.5) / len(u)))
    assert ks < 0.02 + (1 - ok.mean()), ks


def test_smooth_limit_is_the_mirror():
    th = 0.6
    d, w, ok = O.ggx_samples(incoming(th), N, np.full(3, 0.5), 1e-3, 3, 2000)
    mirror = np.array([-np.sin(th), 0.0, np.cos(th)])
    assert ok.all()
    # GGX has long tails (tan theta_m grows as sqrt(u / (1 - u))): bound the
    # bulk of the lobe, not its extreme samples.
    dev = np.linalg.norm(d - mirror, axis=1)
    assert np.percentile(dev, 90) < 1e-2 and np.median(dev) < 3e-3
    # Fresnel with F0 = 0.5 at this angle: the weight is near Schlick's value.
    f = 0.5 + 0.5 * (1 - np.cos(th)) ** 5
    assert np.percentile(np.abs(w[:, 0] / f - 1), 90) < 1e-2
