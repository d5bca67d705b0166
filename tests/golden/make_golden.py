"""Generates the golden fixtures in this directory from the known answers of
aperi-mech's own unit tests (the constructions are restated here; nothing is
read from the reference at run time):

  quadrature_tet4.json         QuadratureTests.cpp:17-125 (reference, x0.78 contraction,
                               translation (0.512,-4.79,103.1), rotation about (1.2,-2.3,1.4)
                               by 0.36 pi, deformed) -> B and w at 1e-12 (:298-315)
  quadrature_hex8_smoothed.json QuadratureTests.cpp:127-296 (smoothed-hex cases, test :353-366)
  material_driver_nh.json      MaterialDriverTest.cpp:38-115: K=2.2e9, mu=1.5e6 neo-Hookean,
                               uniaxial H rows -> Cauchy sigma_ii = 5.24795e6 (1e-6 rel)
  linear_elastic_properties.json LinearElasticPropertiesTest.cpp:16-179

The "deformed" cases use Eigen::Matrix3d::Random() in the reference; here a
seeded numpy draw from the same U[-1, 1] distribution stands in for it.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def rotation(axis, angle):
    """Eigen::AngleAxisd(angle, axis).toRotationMatrix() (Rodrigues)."""
    k = np.asarray(axis, dtype=float)
    k = k / np.linalg.norm(k)
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return math.cos(angle) * np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * np.outer(k, k)


def tet_cases(rng):
    cases = []
    X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    B = np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    w = 1.0 / 6.0
    cases.append(("Reference tetrahedron", X.copy(), B.copy(), w))
    f = 0.78
    X, B, w = X * f, B / f, w * f ** 3
    cases.append(("Contracted reference tetrahedron", X.copy(), B.copy(), w))
    X = X + np.array([0.512, -4.79, 103.1])
    cases.append(("Contracted and translated reference tetrahedron", X.copy(), B.copy(), w))
    R = rotation([1.2, -2.3, 1.4], 0.36 * math.pi)
    X0 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    B0 = np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    cases.append(("Rotated reference tetrahedron", X0 @ R, B0 @ R, 1.0 / 6.0))
    F = rng.uniform(-1, 1, size=(3, 3))
    while np.linalg.det(F) < 0.2:  # right-handed, so the weight stays positive
        F = rng.uniform(-1, 1, size=(3, 3))
    Xd = X0 @ F
    mn, mx = Xd.min(axis=0), Xd.max(axis=0)
    Xd = (Xd - mn) / (mx - mn)
    F = F @ np.diag(1.0 / (mx - mn))
    cases.append(("Deformed tetrahedron", Xd, B0 @ np.linalg.inv(F).T, float(np.linalg.det(F)) / 6.0))
    return cases


def hex_cases(rng):
    cases = []
    X0 = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=float)
    s = 0.25
    B0 = s * np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                       [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=float)
    cases.append(("Reference hexahedron", X0.copy(), B0.copy(), 1.0))
    f = 0.78
    X, B, w = X0 * f, B0 / f, f ** 3
    cases.append(("Contracted reference hexahedron", X.copy(), B.copy(), w))
    cases.append(("Contracted and translated reference hexahedron", X + np.array([0.512, -4.79, 103.1]), B.copy(), w))
    R = rotation([1.2, -2.3, 1.4], 0.36 * math.pi)
    cases.append(("Rotated reference hexahedron", X0 @ R, B0 @ R, 1.0))
    F = rng.uniform(-1, 1, size=(3, 3))
    while np.linalg.det(F) < 0.2:
        F = rng.uniform(-1, 1, size=(3, 3))
    cases.append(("Deformed hexahedron", X0 @ F, B0 @ np.linalg.inv(F).T, float(np.linalg.det(F))))
    sh = 0.2
    Xs = np.array([[sh, 0, 0], [1 + sh, 0, 0], [1 - sh, 1, 0], [-sh, 1, 0],
                   [sh, 0, 1], [1 + sh, 0, 1], [1 - sh, 1, 1], [-sh, 1, 1]], dtype=float)
    b = sh / 2.0
    Bs = np.array([[-s, -(s + b), -s], [s, -(s - b), -s], [s, (s + b), -s], [-s, (s - b), -s],
                   [-s, -(s + b), s], [s, -(s - b), s], [s, (s + b), s], [-s, (s - b), s]])
    cases.append(("Non-planar faced hexahedron", Xs, Bs, 1.0))
    return cases


def dump(name, cases):
    out = [{"name": n, "X": X.tolist(), "B": B.tolist(), "w": float(w)} for n, X, B, w in cases if B is not None]
    (HERE / name).write_text(json.dumps(out, indent=1))


def main():
    rng = np.random.default_rng(42)
    dump("quadrature_tet4.json", tet_cases(rng))
    dump("quadrature_hex8_smoothed.json", hex_cases(rng))
    K, mu = 2.2e9, 1.5e6
    E = 9.0 * mu * K / (3.0 * K + mu)
    nu = (3.0 * K - 2.0 * mu) / (2.0 * (3.0 * K + mu))
    a = -0.2927726653
    Hs = [np.diag([1.0, a, a]), np.diag([a, 1.0, a]), np.diag([a, a, 1.0])]
    (HERE / "material_driver_nh.json").write_text(json.dumps({
        "density": 1.0, "youngs_modulus": E, "poissons_ratio": nu,
        "displacement_gradients": [h.tolist() for h in Hs],
        "expected_cauchy_diagonal": 5.24795e6, "rel_tol": 1e-6}, indent=1))
    E, nu, G, Kb, lam = 200.0, 0.3, 76.92307692307692, 166.66666666666666, 115.38461538461539
    vals = {"youngs_modulus": E, "poissons_ratio": nu, "shear_modulus": G, "bulk_modulus": Kb, "lambda": lam}
    keys = list(vals)
    pairs = [(keys[i], keys[j]) for i in range(5) for j in range(i + 1, 5)]
    (HERE / "linear_elastic_properties.json").write_text(json.dumps({
        "values": vals, "tol": 1e-3, "valid_pairs": pairs,
        "invalid": [{"youngs_modulus": 200.0},
                    {"youngs_modulus": 200.0, "poissons_ratio": 0.3, "shear_modulus": 76.9},
                    {},
                    {"youngs_modulus": -100.0, "poissons_ratio": 0.3},
                    {"youngs_modulus": 100.0, "poissons_ratio": 0.6},
                    {"shear_modulus": 100.0, "lambda": -100.0}]}, indent=1))


if __name__ == "__main__":
    main()
