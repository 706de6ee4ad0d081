"""Seeded synthetic scenes -> target parameters of the tracked problems.

Each generator returns (targets [H, P+1] complex, ground_truth [H, N] real)
for H hypotheses; slot P of every target is 1 (the reference's constant-1
parameter, GPU-HC/magmaHC/Data_Reader.cpp:138-159).  The ground truth is the
unknown vector of the noise-free scene, a real root of the target system.

generalized_3views_4pts (45 parameters, 12 unknowns).  The system
(auto-data-gen-tools/p2c-problems/sys_generalized_3views_4pts.m) states that
the distance between two scene points is the same in all three generalized
cameras:
    | x_a d_a1 - x_b d_b1 + c_ab |^2 = | x_{4+a} d_a2 - x_{4+b} d_b2 + c_ab |^2 ...
with p1..p12 the ray directions of points 1..4 in camera 1 (three per
point), p13..p24 in camera 2, p25..p36 in camera 3, and p37..p45 the ray
origin differences c_12, c_13, c_14 (shared by the cameras); the unknowns
x1..x4, x5..x8, x9..x12 are the depths of the four points along their rays
in cameras 1, 2, 3.  A scene: 4 points uniform in [-1,1]^3 shifted to depth
4..8, 3 cameras with uniform random rotations and N(0,1) translations, ray
origins o_ij = o_1j - c_1i, directions normalised to z = 1 (normalised image
coordinates) with Gaussian noise of sigma = noise_px / focal on x and y.
"""
import numpy as np


def random_rotation(rng):
    """Uniform rotation (Shoemake's quaternion method)."""
    u1, u2, u3 = rng.random(3)
    q = np.array([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def generalized_3views_4pts(n_hyp, seed=0, noise_px=0.5, focal=1000.0, offset_scale=0.2):
    rng = np.random.default_rng(seed)
    P = 45
    targets = np.zeros((n_hyp, P + 1), dtype=np.complex128)
    truth = np.zeros((n_hyp, 12))
    sigma = noise_px / focal
    for h in range(n_hyp):
        while True:
            X = rng.uniform(-1, 1, size=(4, 3))
            X[:, 2] += rng.uniform(4, 8, size=4)
            c1 = offset_scale * rng.normal(size=(4, 3))  # c_1i = o_1j - o_ij, i = 2..4 (row 0 unused)
            c1[0] = 0.0
            dirs = np.zeros((3, 4, 3))
            depth = np.zeros((3, 4))
            ok = True
            for j in range(3):
                R = random_rotation(rng) if j > 0 else np.eye(3)
                t = rng.normal(size=3) if j > 0 else np.zeros(3)
                o1 = offset_scale * rng.normal(size=3)
                for i in range(4):
                    o = o1 - c1[i]
                    Y = R @ X[i] + t - o
                    if Y[2] < 0.5:  # point must be in front of the camera
                        ok = False
                    depth[j, i] = Y[2]
                    d = Y / Y[2]
                    d[:2] += sigma * rng.normal(size=2)
                    dirs[j, i] = d
            if ok:
                break
        p = np.concatenate([dirs[0].reshape(-1), dirs[1].reshape(-1), dirs[2].reshape(-1),
                            c1[1], c1[2], c1[3]])
        targets[h, :P] = p
        targets[h, P] = 1.0
        truth[h] = np.concatenate([depth[0], depth[1], depth[2]])
    return targets, truth


def p3p_td(n_hyp, seed=0):
    """P3P by a total-degree homotopy (problem P3P_TD, 12 parameters, 3 unknowns).

    Returns ((start [P+1], targets [H, P+1]), truth [H, 3]).  One seeded
    unit-modulus gamma per call (the start system gamma (x_k^2 - 1)); per
    hypothesis three points uniform in [-1,1]^3 at depth 4..8 seen from the
    origin: bearings b_i = X_i / |X_i|, c_ij = b_i . b_j, s_ij = |X_i - X_j|^2;
    the true depths |X_i| are a real root of the target system.
    """
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "gen"))
    import make_p3p_td as m
    rng = np.random.default_rng(seed)
    gamma = np.exp(1j * rng.uniform(0.0, 2 * np.pi))
    start = np.append(np.array(m.start_params(gamma), dtype=np.complex128), 1.0)
    targets = np.zeros((n_hyp, 13), dtype=np.complex128)
    truth = np.zeros((n_hyp, 3))
    for h in range(n_hyp):
        X = rng.uniform(-1, 1, size=(3, 3))
        X[:, 2] += rng.uniform(4, 8, size=3)
        d = np.linalg.norm(X, axis=1)
        b = X / d[:, None]
        c = {(i, j): float(b[i] @ b[j]) for (i, j) in m.PAIRS}
        s2 = {(i, j): float(np.sum((X[i] - X[j]) ** 2)) for (i, j) in m.PAIRS}
        targets[h, :12] = m.target_params(c, s2)
        targets[h, 12] = 1.0
        truth[h] = d
    return (start, targets), truth


def small_rotation(rng, max_angle):
    """Rotation about a uniform random axis by an angle uniform in [0, max_angle]."""
    k = rng.normal(size=3)
    k /= np.linalg.norm(k)
    a = rng.uniform(0, max_angle)
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * (K @ K)


def uncalibrated_trifocal_rel_pos_CY(n_hyp, seed=0, noise_px=0.5, outlier_frac=0.3, image_px=1000.0):
    """Trifocal relative pose with an unknown shared focal length (24 parameters, 12 unknowns).

    The system (auto-data-gen-tools/p2c-problems/sys_uncalibrated_trifocal_rel_pos_CY.m)
    equates, for every pair of the 4 points, their distance seen in camera 1
    with camera 2 (f1-f6) and camera 3 (f7-f12), on rays m = (u, v, sqrt(x1)):
        | x_b m_b - x_a m_a |_cam1 = | x_{4+a} n_a - x_{4+b} n_b |_cam2 ...
    Parameters: p1..p4 / p5..p8 the u / v image coordinates of points 1..4 in
    camera 1, p9..p16 in camera 2, p17..p24 in camera 3 (principal point at
    0, units of image_px pixels).  Unknowns: x1 = f^2, x2..x4 the camera-1
    depths of points 2..4 relative to point 1, x5..x8 and x9..x12 the depths
    of points 1..4 in cameras 2 and 3 relative to the same.
    A hypothesis is a minimal sample: each of the 4 correspondences is, with
    probability outlier_frac, replaced in cameras 2 and 3 by a random image
    point.  truth[h] holds the scene's unknowns (meaningful for inlier samples);
    inlier[h] tells which hypotheses are all-inlier.
    """
    rng = np.random.default_rng(seed)
    P = 24
    targets = np.zeros((n_hyp, P + 1), dtype=np.complex128)
    truth = np.zeros((n_hyp, 12))
    inlier = np.zeros(n_hyp, dtype=bool)
    sigma = noise_px / image_px
    for h in range(n_hyp):
        while True:
            f = rng.uniform(0.8, 1.2)
            X = rng.uniform(-1, 1, size=(4, 3))
            X[:, 2] += rng.uniform(4, 8, size=4)
            uv = np.zeros((3, 4, 2))
            z = np.zeros((3, 4))
            ok = True
            for j in range(3):
                R = small_rotation(rng, 0.3) if j > 0 else np.eye(3)
                t = 0.5 * rng.normal(size=3) if j > 0 else np.zeros(3)
                Y = X @ R.T + t
                if np.any(Y[:, 2] < 1.0):
                    ok = False
                z[j] = Y[:, 2]
                uv[j] = f * Y[:, :2] / Y[:, 2:3] + sigma * rng.normal(size=(4, 2))
            if ok:
                break
        out = rng.random(4) < outlier_frac
        for i in np.nonzero(out)[0]:
            for j in (1, 2):
                uv[j, i] = rng.uniform(-0.5, 0.5, size=2)
        inlier[h] = not out.any()
        p = np.concatenate([uv[0, :, 0], uv[0, :, 1], uv[1, :, 0], uv[1, :, 1], uv[2, :, 0], uv[2, :, 1]])
        targets[h, :P] = p
        targets[h, P] = 1.0
        truth[h] = np.concatenate([[f * f], z[0, 1:] / z[0, 0], z[1] / z[0, 0], z[2] / z[0, 0]])
    return targets, truth, inlier


def complex_orthogonal(rng, n=3):
    """Random complex matrix with R^T R = I (Cayley transform of a complex skew matrix)."""
    a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    S = 0.5 * (a - a.T)
    I = np.eye(n)
    return np.linalg.solve(I - S, I + S)


def seed_pair(name, seed=0):
    """A generic complex (solution, parameters) pair with F(x; p) = 0, for monodromy.

    generalized_3views_4pts: a complexified scene -- complex points, complex
    orthogonal camera rotations, complex translations and ray offsets; the
    equations only use bilinear dot products, so the depth identities hold.
    P3P: complex bearings b_i and depths x_i with world points X_i = x_i b_i.
    Returns (x [N] complex, p [P+1] complex with p[P] = 1).
    """
    rng = np.random.default_rng(seed)
    cn = lambda *shape: rng.normal(size=shape) + 1j * rng.normal(size=shape)  # noqa: E731
    if name == "generalized_3views_4pts":
        X = cn(4, 3)
        c1 = cn(4, 3) * 0.3
        c1[0] = 0.0
        dirs = np.zeros((3, 4, 3), dtype=complex)
        depth = np.zeros((3, 4), dtype=complex)
        for j in range(3):
            R = complex_orthogonal(rng) if j > 0 else np.eye(3)
            t = cn(3) if j > 0 else np.zeros(3)
            o1 = cn(3) * 0.3
            for i in range(4):
                Y = R @ X[i] + t - (o1 - c1[i])
                depth[j, i] = Y[2]
                dirs[j, i] = Y / Y[2]
        p = np.concatenate([dirs[0].reshape(-1), dirs[1].reshape(-1), dirs[2].reshape(-1), c1[1], c1[2], c1[3], [1.0]])
        return np.concatenate([depth[0], depth[1], depth[2]]), p
    if name == "P3P":
        b = cn(3, 3)
        x = cn(3)
        X = x[:, None] * b
        return x, np.concatenate([b.reshape(-1), X.reshape(-1), [1.0]])
    raise KeyError(name)


def cayley(r):
    """The unnormalised Cayley matrix M(r) of start-sys-gen/trifocal_2op1p_30x30_monodromySolve.jl:6-11;
    M(r) / (1 + |r|^2) is a rotation."""
    x, y, z = r
    return np.array([[1 + x * x - (y * y + z * z), 2 * (x * y - z), 2 * (x * z + y)],
                     [2 * (x * y + z), 1 + y * y - (x * x + z * z), 2 * (y * z - x)],
                     [2 * (x * z - y), 2 * (y * z + x), 1 + z * z - (x * x + y * y)]])


def trifocal_2op1p_30x30(n_hyp, seed=0, noise_px=0.0, image_px=1000.0, max_angle=0.4):
    """Trifocal relative pose from three points, two of them with curve tangents (33 parameters,
    30 unknowns) -- the system of auto-data-gen-tools/p2c-problems/sys_trifocal_2op1p_30x30.m as
    built by start-sys-gen/trifocal_2op1p_30x30_monodromySolve.jl:13-80.

    Scene: points X_1..X_3 in camera 1 at depth 4-8, unit 3D tangent directions D_1, D_2 at
    X_1, X_2; cameras 2 and 3 with rotations R_v = M(r_v) / s_v (Cayley, s_v = 1 + |r_v|^2,
    angle up to max_angle) and translations T_v ~ N(0, 0.5^2).
    Parameters (the script's flatten order): image points x[p, v, :] for p = 1..3, v = 1..3
    (c1..c18, normalised coordinates), image tangents d[p, v, :] for p = 1, 2 (c19..c30, unit 2D
    directions), then a11 = depth of X_1 in camera 1, e11, e21 = z of D_1, D_2 (c31..c33).
    Unknowns: a21, a31 (camera-1 depths of X_2, X_3), a12, a22, a32, a13, a23, a33 (camera-2/3
    depths times s_v), e12, e13, e22, e23 (z of s_v R_v D_p), u11, u12, u13, u21, u22, u23
    (tangent lengths: D_p in view v = e x_h + u [d; 0]), t2 = s_2 T_2, t3 = s_3 T_3, r2, r3.
    Returns (targets [H, 34] with slot 33 = 1, truth [H, 30]); with noise_px = 0 the truth is an
    exact solution (known-answer test).
    """
    rng = np.random.default_rng(seed)
    sigma = noise_px / image_px
    targets = np.zeros((n_hyp, 34), dtype=np.complex128)
    truth = np.zeros((n_hyp, 30))
    for h in range(n_hyp):
        while True:
            X = rng.uniform(-1, 1, size=(3, 3))
            X[:, 2] += rng.uniform(4, 8, size=3)
            D = rng.normal(size=(2, 3))
            D /= np.linalg.norm(D, axis=1, keepdims=True)
            r = {}
            T = {}
            R = {1: np.eye(3)}
            for v in (2, 3):
                k = rng.normal(size=3)
                k /= np.linalg.norm(k)
                r[v] = np.tan(rng.uniform(0, max_angle) / 2) * k  # Cayley parameter of that rotation
                R[v] = cayley(r[v]) / (1 + r[v] @ r[v])
                T[v] = 0.5 * rng.normal(size=3)
            Y = {1: X}
            for v in (2, 3):
                Y[v] = X @ R[v].T + T[v]
            if all(Y[v][:, 2].min() > 1.0 for v in (1, 2, 3)):
                break
        x = {v: Y[v][:, :2] / Y[v][:, 2:3] for v in (1, 2, 3)}
        d, u, e = {}, {}, {}
        for v in (1, 2, 3):
            for p in (0, 1):
                Dv = R[v] @ D[p]
                g = Dv[:2] - Dv[2] * x[v][p]
                d[p, v] = g / np.linalg.norm(g)
                u[p, v] = np.linalg.norm(g)
                e[p, v] = Dv[2]
        xs = {v: x[v] + sigma * rng.normal(size=x[v].shape) for v in (1, 2, 3)}
        c = []
        for p in range(3):
            for v in (1, 2, 3):
                c += list(xs[v][p])
        for p in (0, 1):
            for v in (1, 2, 3):
                c += list(d[p, v])
        c += [Y[1][0, 2], e[0, 1], e[1, 1]]
        targets[h, :33] = c
        targets[h, 33] = 1.0
        s = {v: 1 + r[v] @ r[v] for v in (2, 3)}
        a = [Y[1][1, 2], Y[1][2, 2]] + [s[2] * Y[2][p, 2] for p in range(3)] + [s[3] * Y[3][p, 2] for p in range(3)]
        ee = [s[2] * e[0, 2], s[3] * e[0, 3], s[2] * e[1, 2], s[3] * e[1, 3]]
        uu = [u[0, 1], s[2] * u[0, 2], s[3] * u[0, 3], u[1, 1], s[2] * u[1, 2], s[3] * u[1, 3]]
        truth[h] = np.concatenate([a, ee, uu, s[2] * T[2], s[3] * T[3], r[2], r[3]])
    return targets, truth


def perturbed_targets(target, n_hyp, seed=0, scale=0.05):
    """Seeded real perturbations of a problem's shipped target parameters (slot P kept at 1).

    Stands in for the scene generator not written here (5-point relative pose):
    real instances near the shipped one.
    """
    rng = np.random.default_rng(seed)
    base = np.asarray(target, dtype=np.complex128)[:-1].real
    out = np.empty((n_hyp, base.size + 1), dtype=np.complex128)
    out[:, :-1] = base[None, :] + scale * rng.normal(size=(n_hyp, base.size))
    out[:, -1] = 1.0
    return out


def targets_for(name, n_hyp, seed, start, shipped_target, **scene):
    """(start params [P+1], targets [H, P+1], truth or None) for a problem's batch.

    ``scene`` is passed to the problem's scene generator (e.g. noise_px)."""
    if name == "generalized_3views_4pts":
        tg, truth = generalized_3views_4pts(n_hyp, seed=seed, **scene)
        return start, tg, truth
    if name == "uncalibrated_trifocal_rel_pos_CY":
        tg, truth, _ = uncalibrated_trifocal_rel_pos_CY(n_hyp, seed=seed, **scene)
        return start, tg, truth
    if name == "P3P_TD":
        (st, tg), truth = p3p_td(n_hyp, seed=seed)
        return st, tg, truth
    if name == "trifocal_2op1p_30x30":
        tg, truth = trifocal_2op1p_30x30(n_hyp, seed=seed, **scene)
        return start, tg, truth
    return start, perturbed_targets(shipped_target, n_hyp, seed=seed), None


GENERATORS = {
    "generalized_3views_4pts": generalized_3views_4pts,
    "uncalibrated_trifocal_rel_pos_CY": uncalibrated_trifocal_rel_pos_CY,
    "P3P_TD": p3p_td,
    "trifocal_2op1p_30x30": trifocal_2op1p_30x30,
}
