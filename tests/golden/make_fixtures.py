"""Regenerate the golden fixtures under tests/golden/.

    python tests/golden/make_fixtures.py decks <path-to-ferrix-checkout>
    python tests/golden/make_fixtures.py box
    python tests/golden/make_fixtures.py beam

`decks` (needs a FerriX checkout, passed explicitly) writes
  decks/<name>.inp.gz   gzip copies of the reference's four test decks
                        (tests/data/*.inp of the FerriX repository), so the
                        GPU parity tests can run where the checkout is absent;
  oracle_<name>.npz     the oracle's full displacement vector after every step
                        of that deck (default initial temperature 20.0, as in
                        tests/calculix_parity.rs:29,91,187,279);
  calculix.json         the CalculiX displacement goldens and tolerances that
                        the reference's tests/calculix_parity.rs asserts.

`box` (no checkout needed) writes
  oracle_c3d20_box.npz  the oracle's FP64 direct solution of the 417,123-DOF
                        C3D20 box that the benchmark solves (ferrix_b200.decks
                        .c3d20_box() with its default seed), plus the deck's
                        SHA-256 so a test can tell when the generator changed.
                        One oracle run: about 70 s on 16 cores, ~10 GB of RAM.

`beam` (no checkout needed) writes
  oracle_c3d4_nlgeom_beam.npz  the oracle's FP64 Cholesky Newton run of the full
                        NLGEOM beam the benchmark times (ferrix_b200.decks
                        .c3d4_nlgeom_beam() with its defaults: 240,000 C3D4,
                        133,623 DOF, E(T), initial temperature gradient, amplitude
                        ramp over 10 increments; default initial temperature 20.0):
                        displacements after the step, increments and Newton
                        iterations, and the deck's SHA-256. About an hour on 8 cores.
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import inp, static_step  # noqa: E402

DECKS = ["C3D4_staticstep", "C3D4_2staticstep", "NLGEOM_test", "C3D20"]

# tests/calculix_parity.rs:65-70, 125-128, 162-165, 219-222, 254-257, 315-319
CALCULIX = {
    "C3D4_staticstep": {"node": 17, "tol": 1e-6, "steps": [[9.356107e-06, -1.313901e-04, 1.719218e-03]]},
    "C3D4_2staticstep": {"node": 17, "tol": 1e-6, "steps": [[9.356107e-06, -1.313901e-04, 1.719218e-03],
                                                            [2.603480e-04, -1.377070e-04, 1.001299e-03]]},
    "NLGEOM_test": {"node": 1, "tol": 5e-3, "steps": [[-9.163880e-02, 3.500324e-01, 1.324598e-01],
                                                      [8.591845e-01, 3.624377e-01, 2.653401e-01]]},
    "C3D20": {"node": 17, "tol": 1e-6, "steps": [[5.752112e-02, -2.497816e-04, -8.074951e-03]]},
}

BOX_FIXTURE = "oracle_c3d20_box.npz"
BEAM_FIXTURE = "oracle_c3d4_nlgeom_beam.npz"


def make_decks(ref: str) -> None:
    os.makedirs(os.path.join(HERE, "decks"), exist_ok=True)
    for name in DECKS:
        src = os.path.join(ref, "tests", "data", name + ".inp")
        with open(src, "rb") as fh:
            raw = fh.read()
        with gzip.GzipFile(os.path.join(HERE, "decks", name + ".inp.gz"), "wb", mtime=0, compresslevel=9) as gz:
            gz.write(raw)
        p = inp.parse_inp_text(raw.decode())
        p.default_initial_temperature = 20.0
        runner = static_step.Runner(p)
        state = static_step.new_state(p)
        timer = inp.SolverTime()
        out = {"node_ids": np.asarray(p.index_to_node_id, dtype=np.int64)}
        for k in range(len(p.steps)):
            runner.solve_step(k, state, timer)
            out[f"step{k + 1}"] = state.displacements.copy()
        np.savez_compressed(os.path.join(HERE, f"oracle_{name}.npz"), **out)
        print(name, "steps", len(p.steps), "dof", len(state.displacements))
    with open(os.path.join(HERE, "calculix.json"), "w") as fh:
        json.dump(CALCULIX, fh, indent=1)


def box_deck() -> str:
    from ferrix_b200 import decks
    return decks.c3d20_box()


def deck_digest(text: str) -> str:
    return hashlib.sha256(text.encode()).hexdigest()


def make_box() -> None:
    text = box_deck()
    t0 = time.perf_counter()
    p = inp.parse_inp_text(text)
    u = static_step.Runner(p).run().displacements
    np.savez_compressed(os.path.join(HERE, BOX_FIXTURE), u=u, deck_sha256=np.array(deck_digest(text)))
    print(BOX_FIXTURE, "dof", len(u), f"{time.perf_counter() - t0:.1f} s")


def beam_deck() -> str:
    from ferrix_b200 import decks
    return decks.c3d4_nlgeom_beam()


def make_beam() -> None:
    text = beam_deck()
    t0 = time.perf_counter()
    p = inp.parse_inp_text(text)
    p.default_initial_temperature = 20.0
    r = static_step.Runner(p)
    u = r.run().displacements
    np.savez_compressed(os.path.join(HERE, BEAM_FIXTURE), u=u, deck_sha256=np.array(deck_digest(text)),
                        increments=np.array(len(r.log)),
                        residual_checks=np.array([len(rec.residuals) for rec in r.log]))
    print(BEAM_FIXTURE, "dof", len(u), "increments", len(r.log), f"{time.perf_counter() - t0:.1f} s")


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "decks":
        make_decks(sys.argv[2])
    elif len(sys.argv) == 2 and sys.argv[1] == "box":
        make_box()
    elif len(sys.argv) == 2 and sys.argv[1] == "beam":
        make_beam()
    else:
        sys.exit(__doc__)
