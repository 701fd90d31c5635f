"""Frequency-domain FWI driver over the engine: the inner loop of the
reference's ``fwi_FD_AC`` (src/AC/fwi_FD_AC.c:229-409) with GRAD_METHOD = 2
(l-BFGS on the device) and LINESEARCH = 2 (the inexact parabolic line search
of ``parabolicls_AC``, src/AC/parabolicls_AC.c:10-230, with
``calc_opt_step``, src/calc_opt_step.c:10-110).

Per iteration, as in the reference: the objective and gradient of the stage's
frequencies over all shots (``gm_grad_obj``, frame-tapered), the descent
direction -grad, the l-BFGS direction (``gm_lbfgs_step``) with the history
rotated once it is full (``rot_LBFGS_vec``) and reset when the direction is
not a descent direction (``check_descent``), the step length from trial
models (``calc_mat_change_wolfe`` in mode 1 + ``obj_AC``), and the model
update (``calc_mat_change_wolfe`` in mode 0).  A stage ends after ITERMAX
iterations, when the relative misfit change over two iterations drops below
PRO, or when no step length is found; the l-BFGS history is cleared between
stages.  Gradient preconditioning (``precond``) and Hessians are left to the
caller (``gm_precond``, ``gm_hessian``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .engine import Engine, Lbfgs, mat_change


@dataclass
class FwiParams:
    itermax: int = 10          # ITERMAX
    nlbfgs: int = 10           # NLBFGS
    eps_scale: float = 0.01    # EPS_SCALE: first trial step = EPS_SCALE max|vp| / max|Hgrad|
    scalefac: float = 2.0      # SCALEFAC
    stepmax: int = 6           # STEPMAX
    pro: float = 0.01          # PRO: stage abort on relative misfit change over two iterations
    vp_low: float = 0.0        # VPLOWERLIM
    vp_up: float = 1e9         # VPUPPERLIM


@dataclass
class FwiLog:
    misfit: list = field(default_factory=list)       # L2 at the start of every iteration
    steps: list = field(default_factory=list)        # eps_scale chosen per iteration
    stage: list = field(default_factory=list)        # stage of every iteration
    obj_calls: int = 0                               # trial misfits of the line searches


def calc_opt_step(l2t, epst):
    """The step at the extremum of the parabola through (epst[i], l2t[i]),
    i = 0..2 (calc_opt_step, src/calc_opt_step.c:55-100)."""
    A = np.array([[1.0, e, e * e] for e in epst], np.float32)
    b = np.array(l2t, np.float32)
    x = np.linalg.solve(A.astype(np.float64), b.astype(np.float64))
    opteps = -x[1] / (2.0 * x[2])
    if 2.0 * x[2] < 0.0 and l2t[1] > l2t[2]:
        opteps = epst[2]
    return float(np.float32(opteps))


def parabolic_line_search(trial, l2, hgrad, vp, p: FwiParams, log: FwiLog | None = None) -> float:
    """parabolicls_AC: trial(alpha) is the misfit of the model updated with
    step alpha (calc_mat_change_wolfe mode 1).  Returns eps_scale (0 when no
    step reduces the misfit within STEPMAX attempts)."""
    alpha = p.eps_scale * float(np.max(vp)) / float(np.max(hgrad))
    l2t = [l2, 0.0, 0.0]
    epst = [0.0, 0.0, 0.0]
    step1 = step2 = 0
    countstep = 0
    its = ite = 1
    while step1 != 1 or step2 != 1:
        for it in range(its, ite + 1):
            l2t[it] = trial(alpha)
            if log is not None:
                log.obj_calls += 1
        if step1 == 0 and l2t[0] <= l2t[1]:
            alpha = alpha / p.scalefac
            countstep += 1
        if step1 == 1 and l2t[1] < l2t[2]:
            epst[2] = alpha
            step2 = 1
        if step1 == 1 and l2t[1] >= l2t[2]:
            epst[2] = alpha
            alpha = alpha + alpha / p.scalefac
            countstep += 1
        if step1 == 0 and l2t[0] > l2t[1]:
            epst[1] = alpha
            step1 = 1
            its = ite = 2
            countstep = 0
            alpha = alpha + alpha / p.scalefac
        if step1 == 0 and countstep > p.stepmax:
            return 0.0
        if step1 == 1 and countstep > p.stepmax:
            step1 = step2 = 1
    return calc_opt_step(l2t, epst)


def run_stage(e: Engine, lb: Lbfgs, vp: np.ndarray, rho: np.ndarray, freqs, xs, ys, rx, ry, obs,
              p: FwiParams, log: FwiLog, stage: int = 1) -> np.ndarray:
    """One workflow stage of fwi_FD_AC on the acoustic engine `e` and the
    device l-BFGS `lb`; returns the updated vp ([NY][NX] float32)."""
    vp = np.array(vp, np.float32, copy=True)
    shape = vp.shape
    hist = {}
    pointer = 1
    lb.zero()
    for it in range(1, p.itermax + 1):
        if pointer > p.nlbfgs:
            lb.rotate()
            pointer = p.nlbfgs
        e.set_model(vp, rho)
        e.factor(freqs)
        grad, _, l2, _ = e.grad_obj(xs, ys, rx, ry, obs)
        grad = grad.reshape(shape)
        gradm = -grad
        hgrad = lb.step(it == 1, pointer, grad, gradm, vp).reshape(shape)
        lb.check_descent(hgrad, grad)

        def trial(alpha):
            vt = mat_change(hgrad, vp, alpha, p.vp_low, p.vp_up, mode=1).reshape(shape)
            e.set_model(vt, rho)
            e.factor(freqs)
            return e.obj(xs, ys, rx, ry, obs)

        eps = parabolic_line_search(trial, l2, hgrad, vp, p, log)
        log.misfit.append(l2)
        log.steps.append(eps)
        log.stage.append(stage)
        hist[it] = l2
        vp = mat_change(hgrad, vp, eps, p.vp_low, p.vp_up, mode=0).reshape(shape)
        diff = abs((hist[it - 2] - hist[it]) / hist[it - 2]) if it > 2 else 1e20
        if it > 1:
            pointer += 1
        if diff <= p.pro or eps < 1e-20 or it == p.itermax:
            break
    return vp
