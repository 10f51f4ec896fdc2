"""The algebra of the mixed form's deviation flux (rusanov_dev32 in
beta1_b200/csrc/mhd_kernels_mixed.cu), restated in numpy.

The kernel evaluates Rusanov(qL, qR; k) - Phi0(k), with Phi0(k) the physical
flux of the reference state q0 through k, from the deviations q - q0, with
the terms rearranged so that no large term is formed and cancelled; Phi0 is
added back in FP64.  In exact arithmetic (here FP64) the rearranged form plus
Phi0 must equal the Rusanov flux itself, and in FP32 its rounding must scale
with the departure from q0 rather than with the flux."""
import numpy as np

GAMMA = 5.0 / 3.0


def prim(q):
    r, u, v, w, p = q
    E = p / (GAMMA - 1.0) + 0.5 * r * (u * u + v * v + w * w)
    return r, np.array([u, v, w]), p, E, np.sqrt(GAMMA * p / r)


def rusanov(qL, qR, k):
    """Reconstruction_Rusanov with piecewise-constant states (the FP64 path)"""
    area = np.linalg.norm(k)
    out = []
    for q in (qL, qR):
        r, u, p, E, c = prim(q)
        U = k @ u
        F = np.array([r * U, r * U * u[0] + k[0] * p, r * U * u[1] + k[1] * p, r * U * u[2] + k[2] * p, U * (E + p)])
        C = np.array([r, r * u[0], r * u[1], r * u[2], E])
        out.append((F, C, abs(U) + c * area))
    (FL, CL, aL), (FR, CR, aR) = out
    return 0.5 * (FL + FR) - 0.5 * max(aL, aR) * (CR - CL)


def deviation_flux(qL, qR, k, q0, dt):
    """rusanov_dev32 with arithmetic type dt, plus Phi0(k) in FP64"""
    r0, u0, p0, E0, _ = prim(q0)
    H = dt(E0 + p0)
    u0t = u0.astype(dt)
    kt = k.astype(dt)
    area = dt(np.linalg.norm(k))
    U0 = kt @ u0t
    dF, dC, rad = [], [], dt(0.0)
    for q in (qL, qR):
        r, u, p, E, c = prim(q)
        dr, dp, dE = dt(r - r0), dt(p - p0), dt(E - E0)
        du = (u - u0).astype(dt)
        uu = u0t + du
        dU = kt @ du
        U = U0 + dU
        dm = dr * U + dt(r0) * dU
        mU0 = dt(r0) * U0
        dF.append(np.array([dm, dm * uu[0] + mU0 * du[0] + kt[0] * dp, dm * uu[1] + mU0 * du[1] + kt[1] * dp,
                            dm * uu[2] + mU0 * du[2] + kt[2] * dp, dU * (H + dE + dp) + U0 * (dE + dp)], dtype=dt))
        dC.append(np.array([dr, dr * uu[0] + dt(r0) * du[0], dr * uu[1] + dt(r0) * du[1], dr * uu[2] + dt(r0) * du[2],
                            dE], dtype=dt))
        rad = max(rad, abs(U) + dt(c) * area)
    dev = dt(0.5) * (dF[0] + dF[1]) - dt(0.5) * rad * (dC[1] - dC[0])
    U0d = k @ u0
    phi = np.array([r0 * U0d, r0 * U0d * u0[0] + k[0] * p0, r0 * U0d * u0[1] + k[1] * p0, r0 * U0d * u0[2] + k[2] * p0,
                    U0d * (E0 + p0)])
    return dev.astype(np.float64) + phi


def cases(n=500, sigma=1e-3, seed=7):
    rng = np.random.default_rng(seed)
    q0 = np.array([1.0, -8.0, 0.0, 0.0, 0.05])
    for _ in range(n):
        qL = q0 + sigma * np.abs(q0).max() * rng.standard_normal(5) * np.array([1e-3, 1, 1, 1, 1e-3])
        qR = q0 + sigma * np.abs(q0).max() * rng.standard_normal(5) * np.array([1e-3, 1, 1, 1, 1e-3])
        yield q0, qL, qR, rng.standard_normal(3)


def test_deviation_form_is_the_rusanov_flux_in_fp64():
    worst = 0.0
    for q0, qL, qR, k in cases():
        ref = rusanov(qL, qR, k)
        got = deviation_flux(qL, qR, k, q0, np.float64)
        worst = max(worst, float(np.abs(got - ref).max() / np.abs(ref).max()))
    assert worst < 1e-14, worst


def test_fp32_rounding_scales_with_the_departure_from_q0():
    dev_err, plain_err = 0.0, 0.0
    for q0, qL, qR, k in cases():
        ref = rusanov(qL, qR, k)
        # errors relative to the momentum flux of the reference state through
        # the face, rho0 |u0|^2 |k| (the flux itself can be small when k is
        # nearly normal to u0)
        scale = q0[0] * (q0[1] ** 2 + q0[2] ** 2 + q0[3] ** 2) * np.linalg.norm(k)
        dev_err = max(dev_err, float(np.abs(deviation_flux(qL, qR, k, q0, np.float32) - ref).max() / scale))
        # the plain FP32 flux: the same arithmetic with q0 = 0 (all of the state is "deviation")
        plain = deviation_flux(qL, qR, k, np.array([1e-300, 0.0, 0.0, 0.0, 1e-300]), np.float32)
        plain_err = max(plain_err, float(np.abs(plain - ref).max() / scale))
    # with departures of ~1e-3 of the flow speed the deviation form is more
    # than two orders of magnitude more accurate than the plain FP32 flux
    # (measured: 2.7e-9 against 6.4e-7)
    assert dev_err < 1e-8, dev_err
    assert plain_err > 100 * dev_err, (plain_err, dev_err)
