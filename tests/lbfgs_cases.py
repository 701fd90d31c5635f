"""Seeded l-BFGS call sequences shared by the CPU pin tests and the GPU
tests: the reference's FWI loop order (src/AC/fwi_FD_AC.c:229-385) --
rotate when the pointer passes NLBFGS, one LBFGS call, pointer + 1 after
every iteration but the first -- over synthetic gradients and models."""
import numpy as np

import oracle as O


def grid(nx=37, ny=29, npml=5, free_surf=0):
    return O.Grid(nx=nx, ny=ny, dh=10.0, npml=npml, free_surf=free_surf)


def sequence(g, nclass, iters, seed):
    """Per iteration: (grad, gradm, model, hess) as [nclass][NY][NX] float32
    (squeezed for one class).  The model drifts along the previous
    iteration's negative gradient, like an FWI update."""
    rng = np.random.default_rng(seed)
    shape = (nclass, g.ny, g.nx)
    model = rng.uniform(1.0, 2.0, shape).astype(np.float32)
    out = []
    for _ in range(iters):
        grad = (rng.standard_normal(shape) * 1e-3).astype(np.float32)
        gradm = (grad * rng.uniform(0.5, 1.5, shape)).astype(np.float32)
        hess = np.exp(rng.uniform(-6, 0, shape)).astype(np.float32)
        sq = (lambda a: a[0]) if nclass == 1 else (lambda a: a)
        out.append((sq(grad), sq(gradm), sq(model.copy()), sq(hess)))
        model = (model - 20.0 * grad + rng.standard_normal(shape).astype(np.float32) * 1e-3).astype(np.float32)
    return out


def run(step, rotate, m, seq, first_of=lambda it: it == 1):
    """Drive step(first, pointer, it, grad, gradm, model, hess) the way the
    reference's loop does; returns the directions of every iteration."""
    pointer = 1
    outs = []
    for it, (grad, gradm, model, hess) in enumerate(seq, start=1):
        if pointer > m:
            rotate()
            pointer = m
        outs.append(step(first_of(it), pointer, it, grad, gradm, model, hess))
        if it > 1:
            pointer += 1
    return outs


def normalise(model, norms):
    """scale_grad(A, 1.0 / MAT_NORM, B) of LBFGS_TE (src/TE/LBFGS_TE.c:31-32):
    the factor is rounded to float, the product formed in float."""
    a = [np.float32(1.0 / np.float64(np.float32(x))) for x in norms]
    return np.stack([(a[c] * model[c]).astype(np.float32) for c in range(2)])
