"""Seeded synthetic `.inp` decks for the linear-static and NLGEOM box workloads.

Every deck is written as Abaqus/CalculiX text in the layout PrePoMax exports
(16 entries per line with trailing-comma continuation, `*Nset` blocks,
`*Step` / `*Static` / `*Boundary` / `*Cload`), so each run goes through the
same `.inp` parser the reference uses (src/solver/parser.rs:111-482).

Workloads (units mm, N, MPa):
  * c3d4_cantilever  - box 10x10x40, 10x10x40 hex cells x 6 Kuhn tets
                       (24,000 C3D4, 4,961 nodes, 14,883 DOF); E=210000,
                       nu=0.3; z=0 face clamped; 1000 N in -y over the z=40 face.
  * c3d20_box        - box 20x20x80, 20x20x80 C3D20 bricks (139,041 nodes,
                       417,123 DOF), interior nodes jittered U(+-10% h), seeded;
                       E=70000, nu=0.33; z=0 clamped; 5000 N in -x over z=80.
  * c3d4_nlgeom_beam - beam 50x10x10, 100x20x20 hex cells -> 240,000 C3D4
                       (44,541 nodes); E(T)=210000-60(T-20) by a two-row
                       *ELASTIC table, *EXPANSION ZERO=20 alpha=1.2e-5, initial
                       temperature 20->220 C along x; x=0 clamped; tip load
                       ramped by an *AMPLITUDE over 10 increments; *STEP, NLGEOM.
  * random_box       - the batched / serving population: box sides U[5,50],
                       cell counts chosen for a log-uniform DOF target,
                       E log-uniform [7e4, 2.1e5], nu U[0.25, 0.35], one face
                       clamped, a random-direction 100-5000 N load on the
                       opposite face, C3D4 or C3D20.
"""
from __future__ import annotations

import io
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

# Kuhn split of a unit cube into 6 tets sharing the (0,0,0)-(1,1,1) diagonal:
# for each axis order (a, b, c): [v0, v0+e_a, v0+e_a+e_b, v111].
_AXIS_ORDERS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]

# Abaqus C3D20 node order in parent coordinates (corners, bottom edges, top edges, verticals).
C3D20_LOCAL = np.array([
    [-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
    [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1],
    [0, -1, -1], [1, 0, -1], [0, 1, -1], [-1, 0, -1],
    [0, -1, 1], [1, 0, 1], [0, 1, 1], [-1, 0, 1],
    [-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], dtype=np.int64)


@dataclass
class BoxMesh:
    xyz: np.ndarray          # (N, 3) float64, node id = index + 1
    conn: np.ndarray         # (E, npe) int64 of node indices (0-based)
    npe: int
    lattice: np.ndarray      # (N, 3) integer lattice coordinates (doubled grid for C3D20)
    dims: Tuple[int, int, int]
    lengths: Tuple[float, float, float]


def tet_box(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float) -> BoxMesh:
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    lat = np.stack([ii.ravel(order="F"), jj.ravel(order="F"), kk.ravel(order="F")], axis=1)
    nid = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)
    xyz = lat * np.array([lx / nx, ly / ny, lz / nz])
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci, cj, ck = ci.ravel(order="F"), cj.ravel(order="F"), ck.ravel(order="F")
    tets = []
    for order in _AXIS_ORDERS:
        p = [np.zeros(3, dtype=np.int64)]
        cur = np.zeros(3, dtype=np.int64)
        for ax in order[:2]:
            cur = cur.copy()
            cur[ax] = 1
            p.append(cur)
        p.append(np.ones(3, dtype=np.int64))
        t = np.stack([nid(ci + q[0], cj + q[1], ck + q[2]) for q in p], axis=1)
        # orient for positive volume (the element routines use |detJ| either way)
        v = np.einsum("ij,ij->i", np.cross(xyz[t[:, 1]] - xyz[t[:, 0]], xyz[t[:, 2]] - xyz[t[:, 0]]),
                      xyz[t[:, 3]] - xyz[t[:, 0]])
        neg = v < 0
        t[neg, 1], t[neg, 2] = t[neg, 2].copy(), t[neg, 1].copy()
        tets.append(t)
    conn = np.stack(tets, axis=1).reshape(-1, 4)
    return BoxMesh(xyz, conn, 4, lat, (nx, ny, nz), (lx, ly, lz))


def hex20_box(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float,
              jitter: float = 0.0, seed: int = 0) -> BoxMesh:
    gx, gy, gz = 2 * nx + 1, 2 * ny + 1, 2 * nz + 1
    ii, jj, kk = np.meshgrid(np.arange(gx), np.arange(gy), np.arange(gz), indexing="ij")
    lat = np.stack([ii.ravel(order="F"), jj.ravel(order="F"), kk.ravel(order="F")], axis=1)
    keep = (lat % 2).sum(axis=1) <= 1
    lat = lat[keep]
    lut = -np.ones(gx * gy * gz, dtype=np.int64)
    lin = lambda a: a[..., 0] + gx * (a[..., 1] + gy * a[..., 2])
    lut[lin(lat)] = np.arange(len(lat))
    h = np.array([lx / nx, ly / ny, lz / nz])
    xyz = lat * (h / 2.0)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        interior = np.all((lat > 0) & (lat < np.array([gx - 1, gy - 1, gz - 1])), axis=1)
        d = rng.uniform(-jitter, jitter, size=(int(interior.sum()), 3)) * h
        xyz[interior] += d
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    base = np.stack([ci.ravel(order="F"), cj.ravel(order="F"), ck.ravel(order="F")], axis=1) * 2
    off = C3D20_LOCAL + 1
    conn = lut[lin(base[:, None, :] + off[None, :, :])]
    assert (conn >= 0).all()
    return BoxMesh(xyz, conn, 20, lat, (nx, ny, nz), (lx, ly, lz))


def _fmt_rows(vals: Sequence[int], per_line: int = 16) -> str:
    out = []
    for i in range(0, len(vals), per_line):
        chunk = ", ".join(str(int(v)) for v in vals[i:i + per_line])
        out.append(chunk + ("," if i + per_line < len(vals) else ""))
    return "\n".join(out)


@dataclass
class DeckSpec:
    mesh: BoxMesh
    materials: List[Tuple[float, float, Optional[float]]]   # (E, nu, T) rows of *ELASTIC
    expansion: Optional[Tuple[float, float]] = None        # (alpha, ZERO)
    clamp_axis: int = 2
    clamp_side: int = 0           # 0: min face, 1: max face
    load_total: Tuple[float, float, float] = (0.0, -1000.0, 0.0)
    nlgeom: bool = False
    static_line: Optional[str] = None
    amplitude: Optional[List[Tuple[float, float]]] = None
    init_temp: Optional[np.ndarray] = None   # per node
    solver: str = "Spooles"
    heading: str = "ferrix-b200 synthetic deck"


def face_nodes(mesh: BoxMesh, axis: int, side: int) -> np.ndarray:
    lat = mesh.lattice[:, axis]
    target = lat.min() if side == 0 else lat.max()
    return np.nonzero(lat == target)[0]


def write_deck(spec: DeckSpec) -> str:
    m = spec.mesh
    s = io.StringIO()
    w = s.write
    w("**\n** " + spec.heading + "\n**\n*Heading\n" + spec.heading + "\n")
    w("**\n** Nodes +++++++++++++++++++++++++++++++++++++++++++++++++++\n**\n*Node\n")
    for i, (x, y, z) in enumerate(m.xyz.tolist()):
        w(f"{i + 1}, {x!r}, {y!r}, {z!r}\n")
    et = "C3D4" if m.npe == 4 else "C3D20"
    w(f"**\n** Elements ++++++++++++++++++++++++++++++++++++++++++++++++\n**\n*Element, Type={et}, Elset=Solid\n")
    for e in range(m.conn.shape[0]):
        w(_fmt_rows([e + 1] + [int(v) + 1 for v in m.conn[e]]) + "\n")
    clamp = face_nodes(m, spec.clamp_axis, spec.clamp_side)
    loaded = face_nodes(m, spec.clamp_axis, 1 - spec.clamp_side)
    w("**\n** Node sets +++++++++++++++++++++++++++++++++++++++++++++++\n**\n*Nset, Nset=Fixed\n")
    w(_fmt_rows(clamp + 1) + "\n")
    w("*Nset, Nset=Loaded\n" + _fmt_rows(loaded + 1) + "\n")
    w("*Elset, Elset=Vol\nSolid\n")
    w("**\n** Materials +++++++++++++++++++++++++++++++++++++++++++++++\n**\n*Material, Name=Mat\n")
    w("*Density\n7.8E-09\n*Elastic\n")
    for e, nu, t in spec.materials:
        w(f"{e!r}, {nu!r}" + (f", {t!r}" if t is not None else "") + "\n")
    if spec.expansion is not None:
        a, zero = spec.expansion
        w(f"*Expansion, Zero={zero!r}\n{a!r}\n")
    w("*Solid section, Elset=Vol, Material=Mat\n")
    if spec.amplitude is not None:
        w("*Amplitude, Name=Ramp\n" + ", ".join(f"{t!r}, {v!r}" for t, v in spec.amplitude) + "\n")
    if spec.init_temp is not None:
        w("*Initial conditions, Type=Temperature\n")
        for i, t in enumerate(spec.init_temp):
            w(f"{i + 1}, {float(t)!r}\n")
    w("**\n** Step-1 ++++++++++++++++++++++++++++++++++++++++++++++++++\n**\n")
    w("*Step, NLGEOM\n" if spec.nlgeom else "*Step\n")
    w(f"*Static, Solver={spec.solver}\n")
    if spec.static_line:
        w(spec.static_line + "\n")
    w("**\n** Boundary conditions +++++++++++++++++++++++++++++++++++++\n**\n")
    w("*Boundary, op=New\n** Name: Fixed-1\n*Boundary\nFixed, 1, 6, 0\n")
    w("**\n** Loads +++++++++++++++++++++++++++++++++++++++++++++++++++\n**\n*Cload, op=New\n")
    w("*Cload" + (", Amplitude=Ramp" if spec.amplitude is not None else "") + "\n")
    n = len(loaded)
    for d in range(3):
        if spec.load_total[d] != 0.0:
            per = float(spec.load_total[d]) / n
            for i in loaded:
                w(f"{i + 1}, {d + 1}, {per!r}\n")
    w("**\n** Field outputs +++++++++++++++++++++++++++++++++++++++++++\n**\n*Node file\nRF, U\n*El file\nS, E, NOE\n")
    w("**\n** End step ++++++++++++++++++++++++++++++++++++++++++++++++\n**\n*End step\n")
    return s.getvalue()


def deck_arrays(spec: DeckSpec) -> dict:
    """The model write_deck(spec) describes, as Project.from_arrays arguments (the
    binary mesh path, fx_model_from_arrays): what the reference parser makes of that
    text, without the text. Node and element ids are 1-based positions; the single
    material is *Elastic rows (E, nu, T; T = 0 when absent) and the optional
    *Expansion (alpha at T = 0, ZERO = reference temperature); the step's solver
    is DIRECT (Spooles); its BCs are the clamped face's nodes x DOFs 1-3 in node
    order, its loads the loaded face's nodes per force component."""
    m = spec.mesh
    n = m.xyz.shape[0]
    ids = np.arange(1, n + 1, dtype=np.int64)
    eids = np.arange(1, m.conn.shape[0] + 1, dtype=np.int64)
    group = (eids, m.conn.astype(np.int64) + 1, np.zeros(len(eids), dtype=np.int32))
    mat = {"name": "MAT", "E": [(0.0 if t is None else t, e) for e, _, t in spec.materials],
           "nu": [(0.0 if t is None else t, nu) for _, nu, t in spec.materials], "alpha": [], "tref": 0.0}
    if spec.expansion is not None:
        mat["alpha"] = [(0.0, spec.expansion[0])]
        mat["tref"] = spec.expansion[1]
    amps = []
    if spec.amplitude is not None:
        amps.append({"time": [t for t, _ in spec.amplitude], "value": [v for _, v in spec.amplitude]})
    clamp = face_nodes(m, spec.clamp_axis, spec.clamp_side)
    loaded = face_nodes(m, spec.clamp_axis, 1 - spec.clamp_side)
    bcs = [(int(i) + 1, d, 0.0, -1, 1) for i in clamp for d in range(3)]
    amp = 0 if spec.amplitude is not None else -1
    loads = [(int(i) + 1, d, float(spec.load_total[d]) / len(loaded), amp, 1)
             for d in range(3) if spec.load_total[d] != 0.0 for i in loaded]
    inc = (1.0, 1.0, 1e-5, 1.0)
    if spec.static_line:
        inc = tuple(float(v) for v in spec.static_line.split(","))
    step = {"nlgeom": spec.nlgeom, "solver": 1 if spec.solver.upper() in ("SPOOLES", "PARDISO", "PASTIX") else 0,
            "increment": inc, "max_increments": 10000, "loads": loads, "bcs": bcs}
    temps = None
    if spec.init_temp is not None:
        temps = {int(i) + 1: float(t) for i, t in enumerate(spec.init_temp)}
    return {"node_ids": ids, "xyz": m.xyz, "c3d4": group if m.npe == 4 else None,
            "c3d20": group if m.npe == 20 else None, "materials": [mat], "amplitudes": amps, "steps": [step],
            "initial_temperatures": temps}


def c3d4_cantilever_spec(nx: int = 10, ny: int = 10, nz: int = 40) -> DeckSpec:
    m = tet_box(nx, ny, nz, 10.0, 10.0, 40.0)
    return DeckSpec(m, [(210000.0, 0.3, None)], clamp_axis=2, load_total=(0.0, -1000.0, 0.0))


def c3d4_cantilever(nx: int = 10, ny: int = 10, nz: int = 40) -> str:
    return write_deck(c3d4_cantilever_spec(nx, ny, nz))


def c3d20_box_spec(nx: int = 20, ny: int = 20, nz: int = 80, seed: int = 2024,
                   lengths=(20.0, 20.0, 80.0)) -> DeckSpec:
    m = hex20_box(nx, ny, nz, *lengths, jitter=0.10, seed=seed)
    return DeckSpec(m, [(70000.0, 0.33, None)], clamp_axis=2, load_total=(-5000.0, 0.0, 0.0))


def c3d20_box(nx: int = 20, ny: int = 20, nz: int = 80, seed: int = 2024, lengths=(20.0, 20.0, 80.0)) -> str:
    return write_deck(c3d20_box_spec(nx, ny, nz, seed, lengths))


def c3d4_nlgeom_beam_spec(nx: int = 100, ny: int = 20, nz: int = 20, tip_load: float = 6.0e4,
                          increments: int = 10) -> DeckSpec:
    m = tet_box(nx, ny, nz, 50.0, 10.0, 10.0)
    temp = 20.0 + 200.0 * m.xyz[:, 0] / 50.0
    dt = 1.0 / increments
    return DeckSpec(m, [(210000.0, 0.3, 20.0), (198000.0, 0.3, 220.0)], expansion=(1.2e-5, 20.0),
                    clamp_axis=0, load_total=(0.0, 0.0, -tip_load), nlgeom=True,
                    static_line=f"{dt!r}, 1.0, 1e-05, {dt!r}", amplitude=[(0.0, 0.0), (1.0, 1.0)],
                    init_temp=temp)


def c3d4_nlgeom_beam(nx: int = 100, ny: int = 20, nz: int = 20, tip_load: float = 6.0e4,
                     increments: int = 10) -> str:
    return write_deck(c3d4_nlgeom_beam_spec(nx, ny, nz, tip_load, increments))


def random_box(rng: np.random.Generator, dof_target: float, npe: int = 4, arrays: bool = False):
    """One member of the batched / serving population; returns (deck, dof), with
    arrays=True (Project.from_arrays arguments of the same model, dof) instead."""
    L = rng.uniform(5.0, 50.0, size=3)
    nodes_target = dof_target / 3.0
    # cells c_i ~ L_i * s with node count ~ prod(c_i + 1) (C3D4) or ~4 prod(c_i) (C3D20)
    vol = float(np.prod(L))
    per_cell = 1.0 if npe == 4 else 4.0
    s = (nodes_target / per_cell / vol) ** (1.0 / 3.0)
    cells = np.maximum(1, np.round(L * s).astype(int))
    e_mod = float(np.exp(rng.uniform(math.log(7.0e4), math.log(2.1e5))))
    nu = float(rng.uniform(0.25, 0.35))
    axis = int(rng.integers(0, 3))
    direction = rng.normal(size=3)
    direction /= np.linalg.norm(direction)
    mag = float(rng.uniform(100.0, 5000.0))
    if npe == 4:
        m = tet_box(int(cells[0]), int(cells[1]), int(cells[2]), *L)
    else:
        m = hex20_box(int(cells[0]), int(cells[1]), int(cells[2]), *L, jitter=0.1, seed=int(rng.integers(1 << 30)))
    spec = DeckSpec(m, [(e_mod, nu, None)], clamp_axis=axis, load_total=tuple(float(v) for v in direction * mag))
    return (deck_arrays(spec) if arrays else write_deck(spec)), 3 * m.xyz.shape[0]


def batch_population(n: int = 256, seed: int = 7, dof_lo: float = 2e3, dof_hi: float = 6e4,
                     c3d20_fraction: float = 0.0, arrays: bool = False) -> List[Tuple[object, int]]:
    """n seeded population members (deck text, or from_arrays arguments with arrays=True:
    the same models, draw for draw)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        target = float(np.exp(rng.uniform(math.log(dof_lo), math.log(dof_hi))))
        npe = 20 if rng.uniform() < c3d20_fraction else 4
        out.append(random_box(rng, target, npe, arrays))
    return out
