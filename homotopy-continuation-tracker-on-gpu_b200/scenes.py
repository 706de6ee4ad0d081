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


GENERATORS = {
    "generalized_3views_4pts": generalized_3views_4pts,
    "P3P_TD": p3p_td,
}
