"""ORACLE — test infrastructure only (never imported by the product path).

Restatement of FerriX's result fields:
  StaticStep::calculate_stress_strain                src/solver/step/static_step.rs:271-379
  Element::calculate_stress_strain_at_local_coords   src/solver/mesh_lib/elements/element.rs:526-566
  build_b_matrix_internal                            src/solver/mesh_lib/elements/element.rs:588-606
  node_local_coords (C3D4 / C3D20)                   src/solver/mesh_lib/elements/c3d4.rs:53-60,
                                                     src/solver/mesh_lib/elements/c3d20.rs:61-84
  Material::update_state (elastic)                   src/solver/material.rs:180-195
  MISES / TRESCA                                     src/solver/io/vtk.rs:262-310

For every element and every one of its nodes: strain = B(xi_node) u_e with the
Jacobian of the undeformed coordinates, minus the thermal strain change
alpha(Tc)(Tc - Tref) - alpha(Ti)(Ti - Tref) on the normal components when the
material has *EXPANSION, stress = D(E(Tc), nu(Tc)) strain; both are summed per
node and divided by the number of elements at the node. The element's D at the
mean element temperature is built too (its only effect is the error when E or
nu is missing). Plain Python loops: small decks only.
"""
from __future__ import annotations

from typing import Tuple

import numpy as np

from .inp import FerrixError, Project

# Abaqus C3D20 node order in local coordinates (c3d20.rs:61-84)
C3D20_NODES = np.array([
    [-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1],
    [0, -1, -1], [1, 0, -1], [0, 1, -1], [-1, 0, -1], [0, -1, 1], [1, 0, 1], [0, 1, 1], [-1, 0, 1],
    [-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], dtype=np.float64)
C3D4_NODES = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)


def c3d20_local_derivatives(p: np.ndarray) -> np.ndarray:
    """dN/d(xi, eta, zeta) of the 20-node serendipity brick at local point p, shape (3, 20)."""
    g = np.zeros((3, 20))
    for a, (xa, ya, za) in enumerate(C3D20_NODES):
        x = p * np.array([xa, ya, za])  # xi*xi_a etc.
        f = 1.0 + x
        if xa != 0 and ya != 0 and za != 0:
            # N = f0 f1 f2 (x0 + x1 + x2 - 2) / 8
            s = x.sum() - 2.0
            for d, cd in enumerate((xa, ya, za)):
                others = np.prod([f[k] for k in range(3) if k != d])
                g[d, a] = cd * others * (s + f[d]) / 8.0
        else:
            m = [k for k, c in enumerate((xa, ya, za)) if c == 0][0]  # the direction along the edge
            cm = 1.0 - p[m] ** 2
            for d, cd in enumerate((xa, ya, za)):
                if d == m:
                    others = np.prod([f[k] for k in range(3) if k != m])
                    g[d, a] = -2.0 * p[m] * others / 4.0
                else:
                    rest = np.prod([f[k] for k in range(3) if k not in (m, d)])
                    g[d, a] = cd * cm * rest / 4.0
    return g


C3D4_DERIVATIVES = np.array([[-1.0, 1.0, 0.0, 0.0], [-1.0, 0.0, 1.0, 0.0], [-1.0, 0.0, 0.0, 1.0]])


def _d_matrix(e: float, nu: float) -> np.ndarray:
    """Isotropic elastic D, Voigt (xx, yy, zz, xy, yz, zx), engineering shear (material.rs:202-230)."""
    f = e / ((1.0 + nu) * (1.0 - 2.0 * nu))
    d = np.zeros((6, 6))
    d[:3, :3] = nu * f
    for k in range(3):
        d[k, k] = (1.0 - nu) * f
        d[3 + k, 3 + k] = (1.0 - 2.0 * nu) / 2.0 * f
    return d


def _b_matrix(dn_global: np.ndarray) -> np.ndarray:
    n = dn_global.shape[1]
    b = np.zeros((6, 3 * n))
    for i in range(n):
        dx, dy, dz = dn_global[:, i]
        c = 3 * i
        b[0, c] = dx
        b[1, c + 1] = dy
        b[2, c + 2] = dz
        b[3, c] = dy
        b[3, c + 1] = dx
        b[4, c + 1] = dz
        b[4, c + 2] = dy
        b[5, c] = dz
        b[5, c + 2] = dx
    return b


def _material_d(mat, temp: float) -> np.ndarray:
    if mat.youngs_modulus is None or mat.poisson_ratio is None:
        raise FerrixError("InvalidModelState", f"missing elastic constants in material '{mat.name}'")
    return _d_matrix(mat.youngs_modulus.interpolate(temp), mat.poisson_ratio.interpolate(temp))


def nodal_stress_strain(p: Project, u: np.ndarray, t_init: np.ndarray, t_cur: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """(S, E), (N, 6) each, in node-index order; nodes of no element stay 0."""
    n = len(p.index_to_node_id)
    xyz = np.asarray([p.nodes[i] for i in p.index_to_node_id], dtype=np.float64).reshape(-1, 3)
    S = np.zeros((n, 6))
    E = np.zeros((n, 6))
    count = np.zeros(n, dtype=np.int64)
    d20 = [c3d20_local_derivatives(q) for q in C3D20_NODES]
    for eid in sorted(p.elements):
        etype, node_ids = p.elements[eid]
        idx = np.array([p.node_id_to_index[nid] for nid in node_ids])
        k = p.element_materials.get(eid)
        if k is None:
            raise FerrixError("InvalidModelState", f"Element {eid} has no material")
        mat = p.materials[k]
        _material_d(mat, float(np.mean(t_cur[idx])))  # the element D at the mean temperature (errors only)
        ue = u.reshape(-1, 3)[idx].ravel()
        xe = xyz[idx]
        for i, node in enumerate(idx):
            dn = C3D4_DERIVATIVES if etype == "C3D4" else d20[i]
            jac = dn @ xe
            if np.linalg.det(jac) == 0.0:
                raise FerrixError("NumericalError", "Singular Jacobian")
            dn_global = np.linalg.inv(jac) @ dn
            strain = _b_matrix(dn_global) @ ue
            tc, ti = float(t_cur[node]), float(t_init[node])
            if mat.thermal_expansion is not None:
                tref = mat.reference_temperature
                delta = (mat.thermal_expansion.interpolate(tc) * (tc - tref)
                         - mat.thermal_expansion.interpolate(ti) * (ti - tref))
                strain[:3] -= delta
            S[node] += _material_d(mat, tc) @ strain
            E[node] += strain
            count[node] += 1
    has = count > 0
    S[has] /= count[has, None]
    E[has] /= count[has, None]
    return S, E


def mises(S: np.ndarray) -> np.ndarray:
    s11, s22, s33, s12, s23, s13 = S.T
    return np.sqrt(((s11 - s22) ** 2 + (s22 - s33) ** 2 + (s33 - s11) ** 2 + 6.0 * (s12 ** 2 + s23 ** 2 + s13 ** 2))
                   / 2.0)


def tresca(S: np.ndarray) -> np.ndarray:
    s11, s22, s33, s12, s23, s13 = S.T
    m = np.stack([np.stack([s11, s12, s13], -1), np.stack([s12, s22, s23], -1), np.stack([s13, s23, s33], -1)], -2)
    ev = np.linalg.eigvalsh(m)
    return ev[:, -1] - ev[:, 0]
