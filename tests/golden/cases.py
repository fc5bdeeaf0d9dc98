"""Netlists of the golden fixtures: the two benchmark circuits plus small edge
cases of the symbolic layer and the NR loop (ragged device mixes, duplicate
stamp slots, a floating source, a capacitor-only node) and the smallest grid
of the uneven-batch family."""
import numpy as np

from karam_b200 import circuits
from karam_b200.circuits import Netlist


def divider():
    """Resistive divider with a current source: linear, one NR step."""
    nl = Netlist()
    nl.vsource(1, 0, 1.0)
    nl.resistor(1, 2, 1e3)
    nl.resistor(2, 0, 2e3)
    nl.isource(0, 2, 1e-4)
    return nl


def floating_source():
    """A voltage source between two non-ground nodes (branch id collision case)."""
    nl = Netlist()
    nl.vsource(1, 0, 1.2)
    nl.vsource(2, 1, 0.5)
    nl.resistor(2, 3, 500.0)
    nl.resistor(3, 0, 1e3)
    nl.diode(3, 0)
    return nl


def parallel_duplicates():
    """Identical devices in parallel: every stamp slot of the pair collides."""
    nl = Netlist()
    nmos = nl.model("NCH", 0, kp=110e-6, vto=0.7, lam=0.04)
    pmos = nl.model("PCH", 1, kp=40e-6, vto=-0.7, lam=0.05)
    nl.vsource(1, 0, 1.8)
    nl.vsource(2, 0, 0.6)
    for _ in range(2):
        nl.mosfet(3, 2, 0, 0, nmos, 2e-6, 0.18e-6)
        nl.mosfet(3, 2, 1, 1, pmos, 4e-6, 0.18e-6)
    nl.resistor(3, 0, 1e5)
    nl.resistor(3, 0, 1e5)
    return nl


def diode_rc():
    """Diode clamp through a series resistor with node caps; node 4 is reached
    only through a capacitor (DC: held by gmin alone)."""
    nl = Netlist()
    nl.vsource(1, 0, 0.0, pulse=(0.0, 1.0, 0.0, 5e-12, 5e-12, 50e-12, 0.0))
    nl.resistor(1, 2, 100.0)
    nl.diode(2, 3)
    nl.resistor(3, 0, 10.0)
    nl.capacitor(2, 0, 1e-15)
    nl.capacitor(3, 4, 1e-15)
    nl.capacitor(4, 0, 1e-15)
    return nl


def grid8():
    """8 x 8 resistor grid with diode clamps and pulsed NMOS loads."""
    return circuits.grid_circuit(8)


def rc_ladder_diodes():
    """RC ladder from a 1 V source with forward-biased diode clamps at every
    fourth node and 1 pF to ground everywhere: no MOSFETs and no diode near
    its conductance floor, so the reference's own AC admittance build and the
    NR-Jacobian rule coincide (the AC pinning case)."""
    nl = Netlist()
    nl.vsource(1, 0, 1.0)
    for k in range(1, 12):
        nl.resistor(k, k + 1, 1e3)
    for k in range(1, 13):
        nl.capacitor(k, 0, 1e-12)
    for k in (4, 8, 12):
        nl.diode(k, 0, 1e-14, 1.0)
    return nl


# AC sweeps of the fixtures: (netlist, input node, f_start, f_stop, points)
AC_CASES = {
    "rc_ladder_diodes": (rc_ladder_diodes, 1, 1e3, 1e11, 17),
    "diode_rc": (diode_rc, 1, 1e6, 1e13, 15),
    "grid8": (grid8, 1, 1e5, 1e11, 13),
    "config2": (circuits.config2, 2, 1e6, 1e12, 13),
}

SMALL = {
    "divider": divider,
    "floating_source": floating_source,
    "parallel_duplicates": parallel_duplicates,
    "diode_rc": diode_rc,
    "grid8": grid8,
}
BENCH = {"config1": circuits.config1, "config2": circuits.config2}

# Larger grids of the uneven-batch family (n = 258, 1026, 4098 unknowns), where
# the level schedules run a CTA per instance. Each fixture holds the symbolic
# layer, DC solutions of two Monte-Carlo instances and a trapezoidal waveform
# of instance 0 (GRID_TRAN), all from the reference-built library.
GRIDS = {"grid16": 16, "grid32": 32, "grid64": 64}
# tiles of the power-grid mesh whose Min-Fill ordering (and, where the
# reference's symbolic factorization finishes in a minute, filled pattern)
# is pinned to the reference build
MESH_ORDERINGS = {"mesh64": 64, "mesh128": 128}
MESH_FILLED = ("mesh64",)


def filled_digest(row_ptr, col):
    """sha256 of a filled pattern's int32 row pointers and columns."""
    import hashlib
    h = hashlib.sha256(np.ascontiguousarray(row_ptr, np.int32).tobytes())
    h.update(np.ascontiguousarray(col, np.int32).tobytes())
    return h.hexdigest()
GRID_TRAN = dict(dt=40e-12, steps=20, max_halvings=6)  # the gate ramp: steps 13-18
GRID_WAVE = {16: [3, 50, 130, 200, 258], 32: [3, 200, 530, 900, 1026],
             64: [3, 900, 2050, 3500, 4098]}

RNG_SEEDS = (circuits.BASE_SEED, circuits.BASE_SEED + 1, circuits.BASE_SEED + 4095, 1)
RNG_COUNT = 64
