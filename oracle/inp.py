"""ORACLE — test infrastructure only (never imported by the product path).

Pure-Python restatement of FerriX's `.inp` preprocessing and keyword parser,
including its quirks, so the oracle builds exactly the model the reference
would build from the same deck text.

Reference (paths relative to the FerriX crate root):
  preprocess_inp / substitute_ccx_solvers   src/solver/parser.rs:903-942
  Parser::parse / parse_keyword / parse_data src/solver/parser.rs:111-510
  parse_node (Node::parse_line)             src/solver/mesh_lib/node.rs:25-35
  Element::parse_line                       src/solver/mesh_lib/elements/element.rs:62-131
  parse_nset / parse_elset                  src/solver/parser.rs:543-602
  parse_elastic / density / expansion       src/solver/parser.rs:604-692
  parse_initial_conditions / depvar         src/solver/parser.rs:694-738
  parse_cload / parse_boundary              src/solver/parser.rs:740-876
  get_keyword_arguments / positional        src/solver/parser.rs:879-894
  Mesh::build_node_mappings                 src/solver/mesh_lib/mesh.rs:35-50
  IncrementData defaults                    src/solver/increment.rs:21-31
  Amplitude::y / interpolate                src/solver/amplitude.rs:39-98
  SolverTime                                src/solver/time.rs:8-63
  SolutionState::initialize                 src/solver/state.rs:47-79

Quirks kept on purpose: only the first data line after *BOUNDARY and
*AMPLITUDE is read; data after an ignored keyword is dropped; DOFs 4-6 are
dropped; a CLOAD on an nset applies the full value to every node; loads and
BCs carry over between steps unless OP=NEW; unknown keywords are errors.
"""
from __future__ import annotations

import bisect
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np


class FerrixError(Exception):
    """Mirror of FerrixError (src/solver/error.rs:12-72); `kind` is the variant."""

    def __init__(self, kind: str, message: str = "", line: int = 0):
        super().__init__(f"{kind}: {message}" + (f" (line {line})" if line else ""))
        self.kind = kind
        self.message = message
        self.line = line


KEYWORDS = {
    "NODE", "ELEMENT", "NSET", "ELSET", "MATERIAL", "ELASTIC", "DENSITY", "SOLID_SECTION",
    "STEP", "STATIC", "BOUNDARY", "CLOAD", "END_STEP", "HEADING", "NODE_FILE", "EL_FILE",
    "AMPLITUDE", "SURFACE", "DLOAD", "DSLOAD", "NODE_PRINT", "EL_PRINT", "INCLUDE",
    "BEAM_SECTION", "EXPANSION", "SHELL_SECTION", "CONDUCTIVITY", "SPECIFIC_HEAT",
    "INITIAL_CONDITIONS", "DEPVAR",
}


_SOLVER_NAMES = {"ITERATIVE CHOLESKY": "ITERATIVE", "ITERATIVE SCALING": "ITERATIVE",
                 "PASTIX": "DIRECT", "PARDISO": "DIRECT", "SPOOLES": "DIRECT"}
_SOLVER_RE = re.compile("|".join(re.escape(k) for k in _SOLVER_NAMES))


def substitute_ccx_solvers(text: str) -> str:
    """parser.rs:930-942: one left-to-right pass replacing non-overlapping matches
    (aho-corasick `replace_all`, standard match semantics; for these five names,
    which never overlap or contain one another, that is the leftmost match), so a
    replacement never forms a new match: "ITERATIVE CHOLESKY SCALING" becomes
    "ITERATIVE SCALING"."""
    return _SOLVER_RE.sub(lambda m: _SOLVER_NAMES[m.group(0)], text)


def preprocess_inp(text: str) -> str:
    out = []
    for raw in text.split("\n"):
        line = raw.strip()
        if not line:
            continue
        line = line.upper()
        line = line + " " if line.endswith(",") else line + "\n"
        if line.startswith("**"):
            continue
        out.append(line)
    return substitute_ccx_solvers("".join(out))


def rust_lines(text: str) -> List[str]:
    """str::lines(): split on \\n, drop one trailing \\r, no trailing empty line."""
    parts = text.split("\n")
    if parts and parts[-1] == "":
        parts.pop()
    return [p[:-1] if p.endswith("\r") else p for p in parts]


def keyword_arguments(line: str) -> Dict[str, Optional[str]]:
    out: Dict[str, Optional[str]] = {}
    for s in line.split(",")[1:]:
        if "=" in s:
            k, v = s.split("=", 1)
            out[k.strip()] = v.strip()
        else:
            out[s.strip()] = None
    return out


def positional_arguments(line: str) -> List[str]:
    return [s.strip() for s in line.split(",")]


def _parse_f64(s: str) -> float:
    """f64::from_str: no surrounding whitespace, no digit separators."""
    if s == "" or "_" in s or s != s.strip():
        raise ValueError(s)
    return float(s)


def _parse_usize(s: str) -> int:
    if s == "" or not s.isdigit() or not s.isascii():
        if s.startswith("+") and s[1:].isdigit() and s[1:].isascii():
            return int(s[1:])
        raise ValueError(s)
    return int(s)


@dataclass
class LUT:
    data: List[Tuple[float, float]] = field(default_factory=list)

    def push(self, t: float, v: float) -> None:
        self.data.append((t, v))
        self.data.sort(key=lambda p: p[0])  # stable, like slice::sort_by

    def interpolate(self, temp: float) -> float:
        d = self.data
        if not d:
            raise AssertionError("Attempted to interpolate an empty LUT")
        if len(d) == 1 or temp <= d[0][0]:
            return d[0][1]
        if temp >= d[-1][0]:
            return d[-1][1]
        lo, hi = 0, len(d) - 1
        while hi - lo > 1:
            mid = lo + (hi - lo) // 2
            if d[mid][0] <= temp:
                lo = mid
            else:
                hi = mid
        t0, v0 = d[lo]
        t1, v1 = d[hi]
        return v0 + (v1 - v0) * ((temp - t0) / (t1 - t0))


@dataclass
class Material:
    name: str
    density: Optional[LUT] = None
    youngs_modulus: Optional[LUT] = None
    poisson_ratio: Optional[LUT] = None
    thermal_expansion: Optional[LUT] = None
    reference_temperature: float = 0.0
    num_depvars: int = 0


@dataclass
class Amplitude:
    total_time: bool = False
    shift_x: float = 0.0
    shift_y: float = 0.0
    times: Optional[List[float]] = None
    values: Optional[List[float]] = None

    def y(self, timer: "SolverTime", origin_step: int, current_step: int) -> float:
        if self.times is not None:
            t = timer.global_ if self.total_time else timer.local
            return amplitude_interpolate(t, self.times, self.values, self.shift_x, self.shift_y)
        if current_step > origin_step:
            return 1.0
        return timer.local / timer.local_max


def amplitude_interpolate(t, times, values, shift_x, shift_y) -> float:
    if not times:
        return 0.0
    tt = t - shift_x
    idx = bisect.bisect_left(times, tt)  # partition_point(|x| x < tt)
    if idx == 0:
        return values[0] + shift_y
    if idx >= len(times):
        return values[len(values) - 1] + shift_y
    t0, t1, v0, v1 = times[idx - 1], times[idx], values[idx - 1], values[idx]
    return v0 + (v1 - v0) / (t1 - t0) * (tt - t0) + shift_y


@dataclass
class Record:
    """A *CLOAD (Load) or *BOUNDARY (BoundaryCondition) entry (boundary_conds.rs)."""
    node_id: int
    dof: int
    value: float
    amplitude: Amplitude
    origin_step: int

    def eval(self, timer: "SolverTime", current_step: int) -> float:
        return self.amplitude.y(timer, self.origin_step, current_step) * self.value


@dataclass
class IncrementData:
    initial_time_increment: float = 1.0
    time_period: float = 1.0
    min_time_increment: float = 1e-5
    max_time_increment: float = 1.0
    max_iterations: int = 10000


@dataclass
class StaticStep:
    solver: str  # "DEFAULT" | "DIRECT" | "ITERATIVE"
    increment: IncrementData
    loads: List[Record]
    bcs: List[Record]
    nlgeom: bool


@dataclass
class SolverTime:
    global_: float = 0.0
    local: float = 0.0
    local_max: float = 1.0

    def new_step(self, max_time: float) -> None:
        self.local = 0.0
        self.local_max = max_time

    def new_increment(self, dt: float) -> None:
        self.global_ += dt
        self.local += dt


@dataclass
class Project:
    nodes: Dict[int, Tuple[float, float, float]] = field(default_factory=dict)
    elements: Dict[int, Tuple[str, Tuple[int, ...]]] = field(default_factory=dict)
    node_sets: Dict[str, List[int]] = field(default_factory=dict)
    element_sets: Dict[str, List[int]] = field(default_factory=dict)
    materials: List[Material] = field(default_factory=list)
    element_materials: Dict[int, int] = field(default_factory=dict)
    steps: List[StaticStep] = field(default_factory=list)
    initial_loads: List[Record] = field(default_factory=list)
    initial_bcs: List[Record] = field(default_factory=list)
    initial_temperatures: Dict[int, float] = field(default_factory=dict)
    default_initial_temperature: float = 0.0
    nodal_output: List[str] = field(default_factory=list)
    element_output: List[str] = field(default_factory=list)
    amplitudes: Dict[str, Amplitude] = field(default_factory=dict)
    index_to_node_id: List[int] = field(default_factory=list)
    node_id_to_index: Dict[int, int] = field(default_factory=dict)

    def build_node_mappings(self) -> None:
        self.index_to_node_id = sorted(self.nodes.keys())
        self.node_id_to_index = {nid: i for i, nid in enumerate(self.index_to_node_id)}

    def index_of(self, node_id: int) -> Optional[int]:
        return self.node_id_to_index.get(node_id)


class Parser:
    def __init__(self, text_preprocessed: str):
        self.lines = rust_lines(text_preprocessed)
        self.p = Project()
        self.current_keyword: Optional[str] = None
        self.line_nr = 0
        self.element_type: Optional[str] = None
        self.elset_name: Optional[str] = None
        self.set_name: Optional[str] = None
        self.is_generate = False
        self.current_step: Optional[StaticStep] = None
        self.step_counter = 0
        self.step_loads: List[Record] = []
        self.step_bcs: List[Record] = []
        self.ic_type: Optional[str] = None
        self.pos = 0

    # peekable iterator over (index, line)
    def _peek(self) -> Optional[str]:
        return self.lines[self.pos] if self.pos < len(self.lines) else None

    def _next(self) -> Optional[str]:
        if self.pos < len(self.lines):
            self.pos += 1
            return self.lines[self.pos - 1]
        return None

    def parse(self) -> Project:
        while self.pos < len(self.lines):
            idx = self.pos
            line = self._next()
            self.line_nr = idx + 1
            if line.startswith("*"):
                self._keyword(line)
                continue
            t = line.strip()
            if not t:
                continue
            if self.current_keyword is not None:
                self._data(t)
        if self.current_step is not None:
            self._finish_step()
        self.p.build_node_mappings()
        return self.p

    def _finish_step(self) -> None:
        st = self.current_step
        st.loads = list(self.step_loads)
        st.bcs = list(self.step_bcs)
        self.p.steps.append(st)
        self.current_step = None

    def _err(self, msg: str) -> FerrixError:
        return FerrixError("ParseError", msg, self.line_nr)

    def _keyword(self, line: str) -> None:
        parts = [s.strip() for s in line.split(",")]
        kw = parts[0][1:].strip().upper()
        key = kw.replace(" ", "_")
        if key not in KEYWORDS:
            raise FerrixError("UnsupportedKeyword", kw, self.line_nr)
        self.current_keyword = key
        ka = keyword_arguments(line)
        if key == "ELEMENT":
            self.element_type = ka.get("TYPE")
            self.elset_name = ka.get("ELSET")
        elif key in ("NSET", "ELSET"):
            self.set_name = ka.get(key)
            self.is_generate = "GENERATE" in ka
        elif key == "MATERIAL":
            name = ka.get("NAME")
            if name is None:
                raise self._err("Material name not found")
            self.p.materials.append(Material(name=name))
        elif key == "EXPANSION":
            if self.p.materials:
                z = ka.get("ZERO")
                if z is not None:
                    try:
                        self.p.materials[-1].reference_temperature = _parse_f64(z)
                    except ValueError:
                        raise self._err("Invalid ZERO value in *EXPANSION")
        elif key == "INITIAL_CONDITIONS":
            t = ka.get("TYPE")
            self.ic_type = t.upper() if t is not None else None
        elif key == "SOLID_SECTION":
            elset = ka.get("ELSET")
            if elset is None:
                raise self._err("Elset not found in *SOLID SECTION")
            mname = ka.get("MATERIAL")
            if mname is None:
                raise self._err("Material not found in *SOLID SECTION")
            midx = next((i for i, m in enumerate(self.p.materials) if m.name == mname), None)
            if midx is None:
                raise FerrixError("MaterialNotFound", mname)
            if elset not in self.p.element_sets:
                raise FerrixError("ElsetNotFound", elset)
            for eid in self.p.element_sets[elset]:
                self.p.element_materials[eid] = midx
        elif key == "STEP":
            if self.step_counter == 0:
                self.step_loads = list(self.p.initial_loads)
                self.step_bcs = list(self.p.initial_bcs)
            self.step_counter += 1
            if self.current_step is not None:
                self._finish_step()
            nlgeom = "NLGEOM" in ka
            inc = ka.get("INC")
            try:
                max_it = _parse_usize(inc) if inc is not None else 10000
            except ValueError:
                max_it = 10000
            nxt = self._peek()
            if nxt is not None and nxt.startswith("*STATIC"):
                ska = keyword_arguments(nxt)
                sv = ska.get("SOLVER")
                if sv is None:
                    solver = "DEFAULT"
                elif sv in ("DIRECT", "ITERATIVE"):
                    solver = sv
                else:
                    raise FerrixError("UnknownSolver", sv)
                self._next()
                incd = IncrementData(max_iterations=max_it)
                dl = self._peek()
                if dl is not None and not dl.startswith("*"):
                    args = positional_arguments(dl)
                    if len(args) >= 4:
                        try:
                            incd.initial_time_increment = _parse_f64(args[0])
                            incd.time_period = _parse_f64(args[1])
                            incd.min_time_increment = _parse_f64(args[2])
                            incd.max_time_increment = _parse_f64(args[3])
                        except ValueError:
                            raise self._err("Invalid increment data")
                    self._next()
                self.current_step = StaticStep(solver, incd, [], [], nlgeom)
        elif key == "END_STEP":
            if self.current_step is not None:
                self._finish_step()
        elif key == "AMPLITUDE":
            name = ka.get("NAME")
            if name is None:
                raise self._err("Amplitude card is missing a Name= argument")
            total = ka.get("TIME") == "TOTAL TIME"
            sx = ka.get("SHIFTX")
            sy = ka.get("SHIFTY")

            def opt_f(s):
                if s is None:
                    return 0.0
                try:
                    return _parse_f64(s)
                except ValueError:
                    return 0.0
            nxt = self._peek()
            if nxt is not None:
                fields = nxt.split(",")
                times = []
                for s in fields[0::2]:
                    try:
                        times.append(_parse_f64(s.strip()))
                    except ValueError:
                        pass
                vals = []
                for s in fields[1::2]:
                    try:
                        vals.append(_parse_f64(s.strip()))
                    except ValueError:
                        raise self._err("Invalid amplitude value")
                self.p.amplitudes[name] = Amplitude(total, opt_f(sx), opt_f(sy), times, vals)
        elif key == "BOUNDARY":
            amp = ka.get("AMPLITUDE")
            if ka.get("OP") == "NEW":
                if self.current_step is not None:
                    self.step_bcs = []
                else:
                    self.p.initial_bcs = []
            nxt = self._peek()
            if nxt is not None and not nxt.startswith("*"):
                self._boundary(nxt, amp)
        elif key == "CLOAD":
            amp = ka.get("AMPLITUDE")
            if ka.get("OP") == "NEW":
                if self.current_step is not None:
                    self.step_loads = []
                else:
                    self.p.initial_loads = []
            while True:
                nxt = self._peek()
                if nxt is None or nxt.startswith("*"):
                    break
                self._next()
                self._cload(nxt, amp)

    def _targets(self, t: str) -> List[int]:
        t = t.strip()
        if t in self.p.node_sets:
            return list(self.p.node_sets[t])
        try:
            return [_parse_usize(t)]
        except ValueError:
            return []

    def _origin(self) -> int:
        return self.step_counter if self.current_step is not None else 0

    def _amp(self, name: Optional[str]) -> Amplitude:
        if name is not None and name in self.p.amplitudes:
            a = self.p.amplitudes[name]
            return Amplitude(a.total_time, a.shift_x, a.shift_y, a.times, a.values)
        return Amplitude()

    def _cload(self, line: str, amp: Optional[str]) -> None:
        parts = [s.strip() for s in line.split(",")]
        if len(parts) < 3:
            return
        try:
            dof = _parse_usize(parts[1])
        except ValueError:
            raise self._err("Invalid DOF")
        try:
            val = _parse_f64(parts[2])
        except ValueError:
            raise self._err("Invalid load value")
        nodes = self._targets(parts[0])
        if 1 <= dof <= 3:
            for nid in nodes:
                rec = Record(nid, dof - 1, val, self._amp(amp), self._origin())
                (self.step_loads if self.current_step is not None else self.p.initial_loads).append(rec)

    def _boundary(self, line: str, amp: Optional[str]) -> None:
        parts = [s.strip() for s in line.split(",")]
        if len(parts) < 2:
            return
        try:
            first = _parse_usize(parts[1])
        except ValueError:
            raise self._err("Invalid first DOF")
        if len(parts) > 2 and parts[2] != "":
            try:
                last = _parse_usize(parts[2])
            except ValueError:
                raise self._err("Invalid last DOF")
        else:
            last = first
        if len(parts) > 3:
            try:
                val = _parse_f64(parts[3])
            except ValueError:
                raise self._err("Invalid boundary value")
        else:
            val = 0.0
        for nid in self._targets(parts[0]):
            for dof in range(first, last + 1):
                if 1 <= dof <= 3:
                    rec = Record(nid, dof - 1, val, self._amp(amp), self._origin())
                    (self.step_bcs if self.current_step is not None else self.p.initial_bcs).append(rec)

    def _data(self, line: str) -> None:
        k = self.current_keyword
        p = self.p
        if k == "NODE":
            f = [s.strip() for s in line.split(",")]
            try:
                if len(f) != 4:
                    raise ValueError
                nid = _parse_usize(f[0])
                xyz = (_parse_f64(f[1]), _parse_f64(f[2]), _parse_f64(f[3]))
            except ValueError:
                raise self._err(f"Invalid node definition: {line}")
            p.nodes[nid] = xyz
        elif k == "ELEMENT":
            if self.element_type is None:
                return
            try:
                nums = [_parse_usize(s.strip()) for s in line.split(",")]
            except ValueError:
                raise FerrixError("ParseError", "Integer conversion failed", 0)
            eid, nodes = nums[0], tuple(nums[1:])
            et = self.element_type
            if et not in ("C3D4", "C3D20"):
                raise FerrixError("ParseError", f"Unknown element definition: {et}", 0)
            if len(nodes) != (4 if et == "C3D4" else 20):
                raise FerrixError("ParseError", f"Wrong node count for {et}", 0)
            if self.elset_name:
                p.element_sets.setdefault(self.elset_name, []).append(eid)
            p.elements[eid] = (et, nodes)
        elif k == "NSET":
            if self.set_name is None or self.is_generate:
                return
            ids = []
            for s in line.split(","):
                s = s.strip()
                if s:
                    try:
                        ids.append(_parse_usize(s))
                    except ValueError:
                        pass
            p.node_sets.setdefault(self.set_name, []).extend(ids)
        elif k == "ELSET":
            if self.set_name is None or self.is_generate:
                return
            ids = []
            for s in line.split(","):
                s = s.strip()
                if s:
                    try:
                        ids.append(_parse_usize(s))
                    except ValueError:
                        pass
            if "," not in line and not ids:
                other = line.strip()
                if other in p.element_sets:
                    add = list(p.element_sets[other])
                    p.element_sets.setdefault(self.set_name, []).extend(add)
            else:
                p.element_sets.setdefault(self.set_name, []).extend(ids)
        elif k in ("ELASTIC", "DENSITY", "EXPANSION"):
            if not p.materials:
                return
            try:
                vals = [_parse_f64(s.strip()) for s in line.split(",")]
            except ValueError:
                raise self._err(f"Invalid {k.lower()} value")
            m = p.materials[-1]
            if k == "ELASTIC":
                if len(vals) >= 2:
                    e, nu = vals[0], vals[1]
                    t = vals[2] if len(vals) >= 3 else 0.0
                    if m.youngs_modulus is None:
                        m.youngs_modulus = LUT()
                    m.youngs_modulus.push(t, e)
                    if m.poisson_ratio is None:
                        m.poisson_ratio = LUT()
                    m.poisson_ratio.push(t, nu)
            else:
                if vals:
                    t = vals[1] if len(vals) >= 2 else 0.0
                    attr = "density" if k == "DENSITY" else "thermal_expansion"
                    if getattr(m, attr) is None:
                        setattr(m, attr, LUT())
                    getattr(m, attr).push(t, vals[0])
        elif k == "INITIAL_CONDITIONS":
            if self.ic_type != "TEMPERATURE":
                return
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 2:
                try:
                    temp = _parse_f64(parts[1])
                except ValueError:
                    raise self._err("Invalid temperature value")
                for nid in self._targets(parts[0]):
                    p.initial_temperatures[nid] = temp
        elif k == "DEPVAR":
            if not p.materials:
                return
            parts = [s.strip() for s in line.split(",")]
            try:
                p.materials[-1].num_depvars = _parse_usize(parts[0])
            except ValueError:
                raise self._err("Invalid DEPVAR value")
        elif k == "NODE_FILE":
            p.nodal_output.extend(s.strip() for s in line.split(","))
        elif k == "EL_FILE":
            p.element_output.extend(s.strip() for s in line.split(","))


def parse_inp_text(text: str) -> Project:
    """Project::from_jobname minus the file read: preprocess + parse."""
    return Parser(preprocess_inp(text)).parse()


def parse_inp_file(path: str) -> Project:
    with open(path, "r") as fh:
        return parse_inp_text(fh.read())


@dataclass
class ModelArrays:
    """Dense numeric view of a Project: node index = rank of the node id."""
    node_ids: np.ndarray          # (N,) int64 sorted
    xyz: np.ndarray               # (N,3) float64
    groups: Dict[int, Tuple[np.ndarray, np.ndarray, np.ndarray]]  # npe -> (elem_ids, conn (E,npe) int32, mat (E,) int32, -1 = none)
    # material pools for the C element routines
    mat_e_off: np.ndarray
    mat_e_len: np.ndarray
    mat_nu_off: np.ndarray
    mat_nu_len: np.ndarray
    mat_a_off: np.ndarray
    mat_a_len: np.ndarray
    mat_tref: np.ndarray
    lut_t: np.ndarray
    lut_v: np.ndarray


def model_arrays(p: Project) -> ModelArrays:
    ids = np.asarray(p.index_to_node_id, dtype=np.int64)
    xyz = np.asarray([p.nodes[i] for i in p.index_to_node_id], dtype=np.float64).reshape(-1, 3)
    groups = {}
    for et, npe in (("C3D4", 4), ("C3D20", 20)):
        eids = sorted(e for e, (t, _) in p.elements.items() if t == et)
        if not eids:
            continue
        conn = np.empty((len(eids), npe), dtype=np.int32)
        mats = np.empty(len(eids), dtype=np.int32)
        for k, eid in enumerate(eids):
            nodes = p.elements[eid][1]
            for a, nid in enumerate(nodes):
                idx = p.node_id_to_index.get(nid)
                if idx is None:
                    raise FerrixError("NodeNotFound", str(nid))
                conn[k, a] = idx
            mats[k] = p.element_materials.get(eid, -1)
        groups[npe] = (np.asarray(eids, dtype=np.int64), conn, mats)
    t_pool: List[float] = []
    v_pool: List[float] = []
    cols = {k: [] for k in ("e_off", "e_len", "nu_off", "nu_len", "a_off", "a_len")}
    tref = []
    for m in p.materials:
        for tag, lut in (("e", m.youngs_modulus), ("nu", m.poisson_ratio), ("a", m.thermal_expansion)):
            cols[tag + "_off"].append(len(t_pool))
            if lut is None:
                cols[tag + "_len"].append(0)
            else:
                cols[tag + "_len"].append(len(lut.data))
                t_pool.extend(t for t, _ in lut.data)
                v_pool.extend(v for _, v in lut.data)
        tref.append(m.reference_temperature)
    i32 = lambda a: np.asarray(a, dtype=np.int32)
    return ModelArrays(ids, xyz, groups, i32(cols["e_off"]), i32(cols["e_len"]), i32(cols["nu_off"]),
                       i32(cols["nu_len"]), i32(cols["a_off"]), i32(cols["a_len"]),
                       np.asarray(tref, dtype=np.float64), np.asarray(t_pool + [0.0], dtype=np.float64),
                       np.asarray(v_pool + [0.0], dtype=np.float64))


def initial_temperatures(p: Project) -> np.ndarray:
    """SolutionState::initialize (state.rs:47-79): default, then *INITIAL CONDITIONS."""
    t = np.full(len(p.index_to_node_id), p.default_initial_temperature, dtype=np.float64)
    for nid, temp in p.initial_temperatures.items():
        idx = p.index_of(nid)
        if idx is not None:
            t[idx] = temp
    return t
