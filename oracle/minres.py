"""MINRES restated from Paige & Saunders (1975), for the oracle (test infrastructure).

The reference solves each Newton correction with ``scipy.sparse.linalg.minres``
(materialite/models/small_strain_fft/small_strain_fft.py:281-299; scipy 1.18.1, an
unpinned third-party dependency).  This is an independent restatement of the published
algorithm (C. C. Paige, M. A. Saunders, "Solution of sparse indefinite systems of linear
equations", SIAM J. Numer. Anal. 12 (1975) 617-629) with the stopping tests that scipy's
implementation applies when ``x0=None``, ``M=None``, ``shift=0``, ``check=False`` and
``maxiter=5n``:

* stop 1 when ||r|| / (||A|| ||x||) <= rtol,
* stop 2 when ||A r|| / (||A|| ||r||) <= rtol,
* stop 3 when ||A|| ||x|| eps >= beta1, stop 4 when cond(A) >= 0.1/eps,
* an early stop when the second Lanczos vector vanishes (beta2 / beta1 <= 10 eps).

``||A||`` is the running Frobenius estimate of the Lanczos tridiagonal matrix and
``cond(A)`` the ratio of the largest to smallest rotation pivot.  ``tests/test_oracle.py``
checks this function against scipy on random symmetric systems.

``atol`` > 0 (not part of the reference) adds the absolute floor that the product's served
requests put on the same tests: stop 1 also when ||r|| <= atol, and no iteration at all when
beta1 <= atol.
"""

import math

import numpy as np


def minres(matvec, b, rtol, maxiter=None, atol=0.0):
    """Solve ``A x = b`` for symmetric ``A`` given as ``matvec``; returns ``(x, iterations)``."""
    b = np.asarray(b, dtype=np.float64)
    n = b.size
    eps = np.finfo(np.float64).eps
    if maxiter is None:
        maxiter = 5 * n
    x = np.zeros(n)
    beta1_sq = float(b @ b)
    if beta1_sq == 0.0:
        return x, 0
    beta1 = math.sqrt(beta1_sq)
    if beta1 <= atol:
        return x, 0

    # Lanczos state: r_prev / r_cur are the unnormalised previous / current vectors.
    r_prev = b
    r_cur = b
    beta_prev = 0.0
    beta = beta1
    # QR-of-tridiagonal state.
    dbar = 0.0
    eps_ln = 0.0
    phibar = beta1
    tnorm2 = 0.0
    gmax = 0.0
    gmin = np.finfo(np.float64).max
    cs, sn = -1.0, 0.0
    w = np.zeros(n)
    w_old = np.zeros(n)
    stop = 0
    itn = 0
    while itn < maxiter:
        itn += 1
        v = r_cur * (1.0 / beta)
        y = matvec(v)
        if itn >= 2:
            y = y - (beta / beta_prev) * r_prev
        alpha = float(v @ y)
        y = y - (alpha / beta) * r_cur
        r_prev, r_cur = r_cur, y
        beta_prev = beta
        beta_sq = float(r_cur @ r_cur)
        if beta_sq < 0.0:
            raise ValueError("non-symmetric matrix")
        beta = math.sqrt(beta_sq)
        tnorm2 += alpha * alpha + beta_prev * beta_prev + beta * beta
        if itn == 1 and beta / beta1 <= 10.0 * eps:
            stop = -1

        # Apply the previous plane rotation, then form the next one.
        eps_prev = eps_ln
        delta = cs * dbar + sn * alpha
        gbar = sn * dbar - cs * alpha
        eps_ln = sn * beta
        dbar = -cs * beta
        root = math.hypot(gbar, dbar)
        gamma = max(math.hypot(gbar, beta), eps)
        cs = gbar / gamma
        sn = beta / gamma
        phi = cs * phibar
        phibar = sn * phibar

        # Search direction and solution update.
        w_new = (v - eps_prev * w_old - delta * w) * (1.0 / gamma)
        w_old, w = w, w_new
        x = x + phi * w

        gmax = max(gmax, gamma)
        gmin = min(gmin, gamma)
        anorm = math.sqrt(tnorm2)
        xnorm = float(np.linalg.norm(x))
        rnorm = phibar
        test1 = math.inf if (xnorm == 0.0 or anorm == 0.0) else rnorm / (anorm * xnorm)
        test2 = math.inf if anorm == 0.0 else root / anorm
        acond = gmax / gmin
        if stop == 0:
            if 1.0 + test2 <= 1.0:
                stop = 2
            if 1.0 + test1 <= 1.0:
                stop = 1
            if itn >= maxiter:
                stop = 6
            if acond >= 0.1 / eps:
                stop = 4
            if anorm * xnorm * eps >= beta1:
                stop = 3
            if test2 <= rtol:
                stop = 2
            if test1 <= rtol:
                stop = 1
            if rnorm <= atol:
                stop = 1
        if stop != 0:
            break
    return x, itn
