"""Oracle restatement of elsa's iterative solvers (TEST INFRASTRUCTURE ONLY).

Only tests/, the smoke check and the benchmark's CPU-baseline arm use this module, as the checker.
It restates the reference solvers on float32 vectors, with the projector given as two callables
(forward A and adjoint A^T, normally oracle.joseph / oracle.joseph_adjoint):

* CGNE       solvers/CGNE.cpp:20-78
* CGLS       solvers/CGLS.cpp:12-91
* Landweber  solvers/LandweberIteration.cpp:26-72, solvers/Landweber.cpp:20-25
* APGD       solvers/APGD.cpp:14-102, proximal_operators/ProximalBoxConstraint.cpp:27-40,
             proximal_operators/ProximalL1.cpp:24-38
* SIRT       solvers/SIRT.cpp:8-45 (Landweber with T A^T M)
* FGM, OGM   solvers/FGM.cpp:33-78, solvers/OGM.cpp:40-95 on LeastSquares (A^T (A x - b))
* SQS        solvers/SQS.cpp:87-170 (ordered subsets, momentum, diagonal preconditioner) and the
             subset splits of projectors/SubsetSampler.cpp:50-103
* powerIterations  solvers/PowerIterations.cpp:10-27

Every solver takes dtype=np.float32 (the reference's float instantiation, the parity target) or
np.float64 (the double instantiation, which shows how far the float32 result itself is from exact
arithmetic). Inner products and norms accumulate in float64 (the reference reduces in float32 with a
thrust transform_reduce whose order depends on the backend, storage/reductions/L2.h:15-33,
DotProduct.h:26-47; a float64 sum is the order-independent limit of those sums). Vector updates
are in dtype like the reference's DataContainer arithmetic; scalars (alpha, beta, t) are rounded
to dtype before they scale a vector, as data_t scalars are in the reference.
"""
import numpy as np

F32_EPS = float(np.finfo(np.float32).eps)


def _caster(dtype):
    return lambda a: np.ascontiguousarray(a, dtype=dtype)


def _sq(a):
    a = np.asarray(a, dtype=np.float64).ravel()
    return float(np.dot(a, a))


def _dot(a, b):
    return float(np.dot(np.asarray(a, dtype=np.float64).ravel(),
                        np.asarray(b, dtype=np.float64).ravel()))


def power_iterations(A, At, domain_size, iterations=5, dtype=np.float32):
    """Largest eigenvalue of A^T A, solvers/PowerIterations.cpp:10-27."""
    _f = _caster(dtype)
    u = np.ones(domain_size, dtype)
    for _ in range(iterations):
        u = _f(At(A(u)))
        u = _f(u / dtype(np.sqrt(_sq(u))))
    v = _f(At(A(u)))
    return _dot(u, v) / np.sqrt(_sq(u))


def cgne(A, At, b, domain_size, iterations, x0=None, dtype=np.float32):
    """CG on A^T A x = A^T b, solvers/CGNE.cpp:20-78. Returns (x, |r|^2 history)."""
    _f = _caster(dtype)
    x = np.zeros(domain_size, dtype) if x0 is None else _f(x0).copy()
    atb = _f(At(b))
    r = _f(atb - _f(At(A(x))))
    c = r.copy()
    kold = _sq(r)
    hist = []
    for _ in range(iterations):
        ac = _f(At(A(c)))
        alpha = dtype(kold / _dot(c, ac))
        x = _f(x + alpha * c)
        r = _f(r - alpha * ac)
        k = _sq(r)
        beta = dtype(k / kold)
        c = _f(r + beta * c)
        kold = k
        hist.append(k)
    return x, hist


def cgls(A, At, b, domain_size, iterations, x0=None, eps=0.0, tol=1e-4, dtype=np.float32):
    """CGLS with damping eps^2, solvers/CGLS.cpp:19-91. Returns (x, |r|^2 history)."""
    _f = _caster(dtype)
    damp = dtype(eps * eps)
    if x0 is not None:
        x = _f(x0).copy()
        s = _f(b - _f(A(x)))
        r = _f(At(s))
        r = _f(r - damp * x)
    else:
        x = np.zeros(domain_size, dtype)
        s = _f(b).copy()
        r = _f(At(s))
    c = r.copy()
    kold = _sq(r)
    hist = []
    for _ in range(iterations):
        if kold < tol:
            break
        q = _f(A(c))
        delta = _sq(q)
        den = delta if damp == 0 else delta + float(damp) * _sq(c)
        alpha = dtype(kold / den)
        x = _f(x + alpha * c)
        s = _f(s - alpha * q)
        r = _f(At(s))
        if damp != 0:
            r = _f(r - damp * x)
        k = _sq(r)
        beta = dtype(k / kold)
        c = _f(r + beta * c)
        kold = k
        hist.append(k)
    return x, hist


def landweber(A, At, b, domain_size, iterations, x0=None, step=None, power_iters=5,
              dtype=np.float32):
    """Landweber iteration x -= step * A^T (A x - b), solvers/LandweberIteration.cpp:26-72.
    Returns (x, step)."""
    _f = _caster(dtype)
    x = np.zeros(domain_size, dtype) if x0 is None else _f(x0).copy()
    if step is None or step <= 0:
        step = 0.9 * (2.0 / power_iterations(A, At, domain_size, power_iters, dtype))
    st = dtype(step)
    for _ in range(iterations):
        res = _f(_f(A(x)) - b)
        x = _f(x - st * _f(At(res)))
    return x, float(step)


def prox(z, mu, kind=0, lower=None, upper=None, sigma=1.0, dtype=np.float32):
    """Proximal operators: 0 identity, 1 box (ProximalBoxConstraint.cpp:27-40),
    2 L1 soft threshold (ProximalL1.cpp:24-38)."""
    _f = _caster(dtype)
    z = _f(z)
    if kind == 1:
        if lower is not None:
            z = np.maximum(z, dtype(lower))
        if upper is not None:
            z = np.minimum(z, dtype(upper))
        return _f(z)
    if kind == 2:
        t = _f(np.abs(z) - dtype(mu) * dtype(sigma))
        t = _f(0.5 * (t + np.abs(t)))
        return _f(np.sign(z) * t)
    return z


def apgd(A, At, b, domain_size, iterations, x0=None, mu=None, epsilon=F32_EPS, kind=0,
         lower=None, upper=None, sigma=1.0, power_iters=5, dtype=np.float32):
    """Accelerated proximal gradient (FISTA), solvers/APGD.cpp:34-102.
    Returns (x, mu, |grad|^2 history)."""
    if mu is None or mu <= 0:
        mu = 0.45 / power_iterations(A, At, domain_size, power_iters, dtype)
    _f = _caster(dtype)
    m = dtype(mu)
    x = np.zeros(domain_size, dtype) if x0 is None else _f(x0).copy()
    x_prev = x.copy()
    y = x.copy()
    t_prev = 1.0
    atb = _f(At(b))

    def gradient(v):
        return _f(_f(At(_f(A(v)))) - atb)

    grad = gradient(y)
    hist = []
    for _ in range(iterations):
        z = _f(y - m * grad)
        x = prox(z, m, kind, lower, upper, sigma, dtype)
        t = (1.0 + np.sqrt(1.0 + 4.0 * t_prev * t_prev)) / 2.0
        coef = dtype((t_prev - 1.0) / t)
        y = _f(x + coef * _f(x - x_prev))
        x_prev = x
        t_prev = t
        g2 = _sq(grad)
        hist.append(g2)
        if g2 <= epsilon:
            break
        grad = gradient(y)
    return x, float(mu), hist


def sirt(A, At, b, domain_size, iterations, x0=None, step=None, power_iters=5,
         dtype=np.float32):
    """SIRT: x -= step * T A^T M (A x - b) with M = 1/(A 1 + 1e-10), T = 1/(A^T 1),
    solvers/SIRT.cpp:20-45 + LandweberIteration.cpp:26-72. Returns (x, step)."""
    _f = _caster(dtype)
    m = _f(1.0 / _f(_f(A(np.ones(domain_size, dtype))) + dtype(1e-10)))
    t = _f(1.0 / _f(At(np.ones(np.asarray(b).size, dtype))))

    def tam_a(v):
        return _f(t * _f(At(_f(m * _f(A(v))))))

    x = np.zeros(domain_size, dtype) if x0 is None else _f(x0).copy()
    if step is None or step <= 0:
        u = np.ones(domain_size, dtype)
        for _ in range(power_iters):
            u = tam_a(u)
            u = _f(u / dtype(np.sqrt(_sq(u))))
        lam = _dot(u, tam_a(u)) / np.sqrt(_sq(u))
        step = 0.9 * (2.0 / lam)
    st = dtype(step)
    for _ in range(iterations):
        res = _f(_f(A(x)) - b)
        x = _f(x - st * _f(t * _f(At(_f(m * res)))))
    return x, float(step)


def _momentum(A, At, b, domain_size, iterations, x0, epsilon, ogm, dtype):
    _f = _caster(dtype)
    x = np.zeros(domain_size, dtype) if x0 is None else _f(x0).copy()
    y_prev = x.copy()
    lip = power_iterations(A, At, domain_size, 20 if ogm else 5, dtype)

    def grad(v):
        return _f(At(_f(_f(A(v)) - b)))

    delta0 = _sq(grad(x))
    theta_prev = 1.0
    hist = []
    for i in range(iterations):
        g = grad(x)
        gl = _f(g / dtype(lip))
        y = _f(x - gl)
        f = 8.0 if (ogm and i == iterations - 1) else 4.0
        theta = 0.5 * (1.0 + np.sqrt(1.0 + f * theta_prev * theta_prev))
        x = _f(y + dtype((theta_prev - 1.0) / theta) * _f(y - y_prev))
        if ogm:
            x = _f(x - dtype(theta_prev / theta) * gl)
        theta_prev = theta
        y_prev = y
        g2 = _sq(g)
        hist.append(g2)
        if g2 <= epsilon * epsilon * delta0:
            break
    return x, lip, hist


def fgm(A, At, b, domain_size, iterations, x0=None, epsilon=F32_EPS, dtype=np.float32):
    """Fast gradient method on 0.5 |A x - b|^2, solvers/FGM.cpp:33-78. Returns
    (x, lipschitz, |grad|^2 history)."""
    return _momentum(A, At, b, domain_size, iterations, x0, epsilon, False, dtype)


def ogm(A, At, b, domain_size, iterations, x0=None, epsilon=F32_EPS, dtype=np.float32):
    """Optimized gradient method on 0.5 |A x - b|^2, solvers/OGM.cpp:40-95."""
    return _momentum(A, At, b, domain_size, iterations, x0, epsilon, True, dtype)


def sqs(A, At, b, domain_size, iterations, x0=None, subsets=None, momentum=True,
        epsilon=F32_EPS, precond=None, dtype=np.float32):
    """SQS on 0.5 |A x - b|^2, solvers/SQS.cpp:87-170. subsets: list of (A_m, At_m, b_m) for the
    ordered-subset mode (None: the full problem); precond: diagonal applied to each gradient.
    As in the reference, z is the same vector as x: the momentum update overwrites x, and
    nextT = 1 + sqrt(1 + 4 t t) / 2. Returns (x, |g|^2 history, stopped early)."""
    c = _caster(dtype)
    one = dtype(1)
    x = c(np.zeros(domain_size)) if x0 is None else c(x0).copy()
    b = c(b)
    grad = lambda A_, At_, b_, v: c(At_(c(c(A_(v)) - b_)))  # noqa: E731
    threshold = _sq(grad(A, At, b, x)) * epsilon * epsilon
    D = c(At(c(A(c(np.ones(domain_size))))))
    with np.errstate(divide="ignore"):
        D = c(one / D)
    prev_t, t = one, one
    prev_x = x.copy()
    parts = subsets if subsets else [(A, At, b)]
    n_sub = dtype(len(parts))
    history = []
    for _ in range(iterations):
        for (Am, Atm, bm) in parts:
            g = grad(Am, Atm, c(bm), x)
            if precond is not None:
                g = c(c(precond) * g)
            g2 = _sq(g)
            history.append(g2)
            if momentum:
                next_t = dtype(one + dtype(np.sqrt(dtype(one + dtype(dtype(4) * t) * t))) /
                               dtype(2))
                x = c(x - c(n_sub * c(D * g)))
                x = c(x + c(dtype(prev_t / next_t) * c(x - prev_x)))
            else:
                x = c(x - c(n_sub * c(D * g)))
            if g2 <= threshold:
                if not subsets or _sq(grad(A, At, b, x)) <= threshold:
                    return x, history, True
            if momentum:
                prev_t, t = t, next_t
                prev_x = x.copy()
    return x, history, False


def subset_split_round_robin(indices, n_subsets):
    """SubsetSampler::splitRoundRobin, projectors/SubsetSampler.cpp:56-69."""
    out = [[] for _ in range(n_subsets)]
    for i, v in enumerate(indices):
        out[i % n_subsets].append(int(v))
    return out


def subset_split_rotational(dim, poses, n_subsets):
    """SubsetSampler::splitRotationalClustering, projectors/SubsetSampler.cpp:71-103: pose
    indices sorted by the rotation angle to the first pose, then round robin. Rotation blocks
    come from the extrinsic matrix [R | t] of the 40-float pose records (offset 27, row stride
    dim + 1); products and the trace in float32 with sequential sums, the angle as the reference
    computes it (2D atan2 in float, 3D acos in double). Python's sort is stable where the
    reference's std::sort is not: the two agree whenever the angles are distinct."""
    P = np.asarray(poses, np.float32).reshape(-1, 40)
    R = [P[i, 27:27 + dim * (dim + 1)].reshape(dim, dim + 1)[:, :dim] for i in range(len(P))]

    def prod(a, b, i, j):
        acc = np.float32(a[i, 0] * b[j, 0])
        for k in range(1, dim):
            acc = np.float32(acc + np.float32(a[i, k] * b[j, k]))
        return acc

    def dist(g):
        if dim == 2:
            return float(np.arctan2(prod(R[0], g, 1, 0), prod(R[0], g, 0, 0)))
        tr = np.float32(np.float32(prod(R[0], g, 0, 0) + prod(R[0], g, 1, 1)) + prod(R[0], g, 2, 2))
        return float(np.arccos((float(tr) - 1.0) / 2.0))

    idx = sorted(range(len(P)), key=lambda i: dist(R[i]))
    return subset_split_round_robin(idx, n_subsets)
