"""Netlists of the benchmark circuit families and the Monte-Carlo sampler.

The netlist object mirrors the global block of the reference's TensorNetlist
(netlist/circuit.h:1056-1216) in insertion order and converts to the flat
``karam_netlist`` struct of include/karam.h. Voltage sources are the
reference's Norton sources (G = 1e3 S, physics/circuitsim.h:2441-2467).

Monte-Carlo parameters come from a restatement of the reference's portable
generator (math/portable_rng.h:15-95: PCG32 with the default stream, Box-Muller
normal with a cached spare), vectorised across instances. Sampled KP/VTO are
rounded to FP32 so the device can store them in FP32 exactly.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A

# Level-1 model cards of the inverter-chain family of the benchmark circuits.
NMOS_CARD = dict(kp=110e-6, vto=0.7, lam=0.04)
PMOS_CARD = dict(kp=40e-6, vto=-0.7, lam=0.05)
NMOS_WL = (2e-6, 0.18e-6)
PMOS_WL = (4e-6, 0.18e-6)


@dataclass
class Netlist:
    n_nodes: int = 0
    temp_k: float = 300.15
    vsrc: list = field(default_factory=list)     # (pos, neg, dc, kind, pulse7)
    isrc: list = field(default_factory=list)     # (pos, neg, amp)
    res: list = field(default_factory=list)      # (n1, n2, ohm)
    cap: list = field(default_factory=list)      # (n1, n2, farad)
    dio: list = field(default_factory=list)      # (a, c, is, n, vt, model)
    mos: list = field(default_factory=list)      # (d, g, s, b, w, l, model)
    models: list = field(default_factory=list)   # (name, type, kp, vto, lam)
    _keep: list = field(default_factory=list, repr=False)
    _struct: object = field(default=None, repr=False)

    # -- builders ---------------------------------------------------------
    def _touch(self, *nodes):
        self._struct = None
        self.n_nodes = max([self.n_nodes, *nodes])

    def model(self, name, mtype, kp=math.nan, vto=math.nan, lam=math.nan):
        self._struct = None
        self.models.append((name, mtype, kp, vto, lam))
        return len(self.models) - 1

    def vsource(self, pos, neg, dc, pulse=None):
        kind = A.SRC_PULSE if pulse is not None else A.SRC_DC
        self.vsrc.append((pos, neg, float(dc), kind, tuple(pulse or (0.0,) * 7)))
        self._touch(pos, neg)
        return len(self.vsrc) - 1

    def isource(self, pos, neg, amp):
        self.isrc.append((pos, neg, float(amp)))
        self._touch(pos, neg)

    def resistor(self, n1, n2, ohm):
        self.res.append((n1, n2, float(ohm)))
        self._touch(n1, n2)

    def capacitor(self, n1, n2, farad):
        self.cap.append((n1, n2, float(farad)))
        self._touch(n1, n2)

    def diode(self, a, c, i_s=1e-14, n=1.0, vt=0.02585, model=-1):
        self.dio.append((a, c, float(i_s), float(n), float(vt), model))
        self._touch(a, c)

    def mosfet(self, d, g, s, b, model, w, l):
        self.mos.append((d, g, s, b, float(w), float(l), model))
        self._touch(d, g, s, b)

    def new_node(self):
        self._struct = None
        self.n_nodes += 1
        return self.n_nodes

    # -- conversion -------------------------------------------------------
    def arrays(self):
        """Numpy arrays of every device table (netlist order)."""
        i32 = lambda xs: np.ascontiguousarray(np.array(xs, dtype=np.int32).reshape(-1))
        f64 = lambda xs: np.ascontiguousarray(np.array(xs, dtype=np.float64).reshape(-1))
        out = {}
        v = self.vsrc
        out["vs_pos"] = i32([x[0] for x in v]); out["vs_neg"] = i32([x[1] for x in v])
        out["vs_dc"] = f64([x[2] for x in v]); out["vs_kind"] = i32([x[3] for x in v])
        out["vs_pulse"] = f64([x[4] for x in v])
        out["is_pos"] = i32([x[0] for x in self.isrc]); out["is_neg"] = i32([x[1] for x in self.isrc])
        out["is_amp"] = f64([x[2] for x in self.isrc])
        out["r_n1"] = i32([x[0] for x in self.res]); out["r_n2"] = i32([x[1] for x in self.res])
        out["r_ohm"] = f64([x[2] for x in self.res])
        out["c_n1"] = i32([x[0] for x in self.cap]); out["c_n2"] = i32([x[1] for x in self.cap])
        out["c_farad"] = f64([x[2] for x in self.cap])
        d = self.dio
        out["d_anode"] = i32([x[0] for x in d]); out["d_cathode"] = i32([x[1] for x in d])
        out["d_is"] = f64([x[2] for x in d]); out["d_n"] = f64([x[3] for x in d])
        out["d_vt"] = f64([x[4] for x in d]); out["d_model"] = i32([x[5] for x in d])
        m = self.mos
        for k, name in enumerate(("m_d", "m_g", "m_s", "m_b")):
            out[name] = i32([x[k] for x in m])
        out["m_w"] = f64([x[4] for x in m]); out["m_l"] = f64([x[5] for x in m])
        out["m_model"] = i32([x[6] for x in m])
        out["model_type"] = i32([x[1] for x in self.models])
        out["model_kp"] = f64([x[2] for x in self.models])
        out["model_vto"] = f64([x[3] for x in self.models])
        out["model_lambda"] = f64([x[4] for x in self.models])
        return out

    def as_struct(self) -> A.KaramNetlist:
        """The karam_netlist view; cached, and valid while this object lives."""
        if self._struct is not None:
            return self._struct
        a = self.arrays()
        names = (C.c_char_p * max(1, len(self.models)))(*[x[0].encode() for x in self.models])
        self._keep = [a, names]
        s = A.KaramNetlist()
        s.n_nodes = self.n_nodes
        s.temp_k = self.temp_k
        s.n_vsrc = len(self.vsrc); s.n_isrc = len(self.isrc); s.n_res = len(self.res)
        s.n_cap = len(self.cap); s.n_dio = len(self.dio); s.n_mos = len(self.mos)
        s.n_models = len(self.models)
        for key, arr in a.items():
            ctype = C.c_int32 if arr.dtype == np.int32 else C.c_double
            setattr(s, key, A.ptr(arr if arr.size else None, ctype))
        s.model_name = C.cast(names, C.POINTER(C.c_char_p))
        self._struct = s
        return s

    @property
    def n_mos(self):
        return len(self.mos)


# ---------------------------------------------------------------------------
# circuit families
# ---------------------------------------------------------------------------
def inverter_chain(stages=32, vdd=1.8, vin=0.9, clamps=0, node_cap=0.0,
                   vin_pulse=None, clamp_rs=10.0, clamp_is=1e-14, clamp_n=1.0):
    """CMOS inverter chain of level-1 MOSFETs.

    Node 1 = VDD, node 2 = IN, nodes 3.. = stage outputs. ``clamps`` diode
    clamps to ground (anode at ground, cathode on an internal node reached
    through RS from every (stages/clamps)-th output) and ``node_cap`` farads
    from every output and internal node to ground.
    """
    nl = Netlist()
    nmod = nl.model("NMOS", A.MODEL_NMOS, NMOS_CARD["kp"], NMOS_CARD["vto"], NMOS_CARD["lam"])
    pmod = nl.model("PMOS", A.MODEL_PMOS, PMOS_CARD["kp"], PMOS_CARD["vto"], PMOS_CARD["lam"])
    VDD, IN = 1, 2
    nl.vsource(VDD, 0, vdd)
    nl.vsource(IN, 0, vin if vin_pulse is None else vin_pulse[0], pulse=vin_pulse)
    outs = []
    prev = IN
    for k in range(stages):
        out = 3 + k
        nl.mosfet(out, prev, VDD, VDD, pmod, *PMOS_WL)
        nl.mosfet(out, prev, 0, 0, nmod, *NMOS_WL)
        outs.append(out)
        prev = out
    internal = []
    if clamps:
        step = stages // clamps
        for j in range(clamps):
            tap = outs[(j + 1) * step - 1]
            node = nl.new_node()
            nl.resistor(tap, node, clamp_rs)
            nl.diode(0, node, clamp_is, clamp_n)
            internal.append(node)
    if node_cap > 0.0:
        for node in outs + internal:
            nl.capacitor(node, 0, node_cap)
    return nl


def config1():
    """32-stage chain, VIN held at 0.9 V: single-instance DC operating point (n = 34)."""
    return inverter_chain(stages=32, vdd=1.8, vin=0.9)


RAMP_PULSE = (0.0, 1.8, 0.0, 200e-12, 200e-12, 1e-9, 0.0)


def config2():
    """256-stage chain + 64 diode clamps (IS 1e-14, N 1, RS 10 ohm) + 1 fF node
    caps, input PULSE 0 -> 1.8 V with a 200 ps rise (n = 322)."""
    return inverter_chain(stages=256, vdd=1.8, clamps=64, node_cap=1e-15,
                          vin_pulse=RAMP_PULSE)


GRID_GATE_PULSE = (0.0, 1.8, 0.5e-9, 0.2e-9, 0.2e-9, 2e-9, 5e-9)
GRID_SIZES = (8, 64)


def grid_circuit(N, seed=None, vdd=1.0, gate_pulse=GRID_GATE_PULSE):
    """N x N resistor grid of the uneven-batch family.

    Node 1 = VDD (``vdd`` volts), node 2 = the loads' gate net (PULSE), grid
    node (i, j) = 3 + i N + j. Segment resistors are log-uniform in
    10 ohm..10 kohm, each grid node has 1 pF to ground, the four corners are
    fed from VDD through 1 ohm pads, 10 % of the nodes carry a diode clamp to
    ground (anode at ground, IS 1e-14, N 1) and 5 % a level-1 NMOS current
    load (drain on the node, gate on the pulsed net, W/L 2u/0.18u). The draws
    come from PortableRNG(seed), seed = BASE_SEED + N by default, so every
    grid of one size is the same circuit; Monte-Carlo instances vary the
    loads' KP/VTO.
    """
    if N < 2:
        raise ValueError("grid needs N >= 2")
    rng = PCG32(np.array([BASE_SEED + N if seed is None else seed], dtype=np.uint64))
    uniform = lambda: float(rng.next()[0]) / 4294967296.0
    nl = Netlist()
    nmod = nl.model("NMOS", A.MODEL_NMOS, NMOS_CARD["kp"], NMOS_CARD["vto"], NMOS_CARD["lam"])
    VDD, GATE = 1, 2
    node = lambda i, j: 3 + i * N + j
    nl.vsource(VDD, 0, vdd)
    nl.vsource(GATE, 0, gate_pulse[0], pulse=gate_pulse)
    for i in range(N):
        for j in range(N):
            if j + 1 < N:
                nl.resistor(node(i, j), node(i, j + 1), 10.0 ** (1.0 + 3.0 * uniform()))
            if i + 1 < N:
                nl.resistor(node(i, j), node(i + 1, j), 10.0 ** (1.0 + 3.0 * uniform()))
    for i, j in ((0, 0), (0, N - 1), (N - 1, 0), (N - 1, N - 1)):
        nl.resistor(VDD, node(i, j), 1.0)
    for i in range(N):
        for j in range(N):
            nl.capacitor(node(i, j), 0, 1e-12)
    for k in range(N * N):
        u = uniform()
        if u < 0.10:
            nl.diode(0, 3 + k, 1e-14, 1.0)
        elif u < 0.15:
            nl.mosfet(3 + k, GATE, 0, 0, nmod, *NMOS_WL)
    return nl


MESH_GATE_PULSE = (0.0, 1.0, 0.1e-9, 0.05e-9, 0.05e-9, 0.4e-9, 1e-9)  # 1 ns period


def power_grid_mesh(N, seed=None, vdd=1.0, pad_pitch=64, load_fraction=20_000 / 1_048_576,
                    gate_pulse=MESH_GATE_PULSE):
    """N x N power-grid mesh of the large single-instance family (the
    1024 x 1024 mesh at N = 1024; smaller N are tiles of the same
    construction).

    Node 1 = VDD (``vdd`` volts), node 2 = the loads' gate net (PULSE, 1 ns
    period), mesh node (i, j) = 3 + i N + j. Segment resistors are uniform in
    0.1..1 ohm, each mesh node has 10 fF to ground, every pad_pitch-th border
    node (the corners included) is fed from VDD through 1 ohm, and a fraction
    load_fraction of the nodes (20 k of 1 M at full size), drawn at random,
    carries a level-1 NMOS load (drain on the node, gate on the pulsed net,
    W/L 2u/0.18u). Draws come from PortableRNG(seed), seed = BASE_SEED +
    10,000,000 + N by default.
    """
    if N < 2:
        raise ValueError("mesh needs N >= 2")
    rng = PCG32(np.array([BASE_SEED + 10_000_000 + N if seed is None else seed], dtype=np.uint64))
    uniform = lambda: float(rng.next()[0]) / 4294967296.0
    nl = Netlist()
    nmod = nl.model("NMOS", A.MODEL_NMOS, NMOS_CARD["kp"], NMOS_CARD["vto"], NMOS_CARD["lam"])
    VDD, GATE = 1, 2
    node = lambda i, j: 3 + i * N + j
    nl.vsource(VDD, 0, vdd)
    nl.vsource(GATE, 0, gate_pulse[0], pulse=gate_pulse)
    for i in range(N):
        for j in range(N):
            if j + 1 < N:
                nl.resistor(node(i, j), node(i, j + 1), 0.1 + 0.9 * uniform())
            if i + 1 < N:
                nl.resistor(node(i, j), node(i + 1, j), 0.1 + 0.9 * uniform())
    border = set()
    for k in range(0, N, pad_pitch):
        border.update({(0, k), (N - 1, k), (k, 0), (k, N - 1)})
    border.update({(0, N - 1), (N - 1, 0), (N - 1, N - 1)})
    for i, j in sorted(border):
        nl.resistor(VDD, node(i, j), 1.0)
    for i in range(N):
        for j in range(N):
            nl.capacitor(node(i, j), 0, 10e-15)
    for k in range(N * N):
        if uniform() < load_fraction:
            nl.mosfet(3 + k, GATE, 0, 0, nmod, *NMOS_WL)
    return nl


def config3_sizes(n_instances=2048, first_instance=0):
    """Grid size N ~ U{8..64} of each instance of the uneven batch: one
    PortableRNG draw per instance, seeded BASE_SEED + 5,000,000 + instance."""
    ids = np.arange(first_instance, first_instance + n_instances, dtype=np.uint64)
    rng = PCG32(ids + np.uint64(BASE_SEED + 5_000_000))
    lo, hi = GRID_SIZES
    return (lo + (rng.next().astype(np.uint64) % np.uint64(hi - lo + 1))).astype(np.int64)


# ---------------------------------------------------------------------------
# Monte-Carlo sampling (math/portable_rng.h:15-95)
# ---------------------------------------------------------------------------
_PCG_MULT = np.uint64(6364136223846793005)
_PCG_STREAM = np.uint64(0xDA3E39CB94B95BDB)
BASE_SEED = 20261203


class PCG32:
    """PortableRNG over a vector of seeds (one generator per instance)."""

    def __init__(self, seeds):
        seeds = np.asarray(seeds, dtype=np.uint64)
        with np.errstate(over="ignore"):
            self.inc = np.full_like(seeds, (_PCG_STREAM << np.uint64(1)) | np.uint64(1))
            self.state = np.zeros_like(seeds)
            self.next()
            self.state = self.state + seeds
            self.next()

    def next(self):
        with np.errstate(over="ignore"):
            old = self.state
            self.state = old * _PCG_MULT + self.inc
            xorshifted = (((old >> np.uint64(18)) ^ old) >> np.uint64(27)).astype(np.uint32)
            rot = (old >> np.uint64(59)).astype(np.uint32)
            left = ((~rot + np.uint32(1)) & np.uint32(31))
            return (xorshifted >> rot) | (xorshifted << left)


def normal_pairs(rng: PCG32):
    """One Box-Muller draw: (cos sample, cached sin sample) per generator."""
    u1 = rng.next().astype(np.float64) / 4294967296.0
    u2 = rng.next().astype(np.float64) / 4294967296.0
    u1 = np.where(u1 < 1e-15, 1e-15, u1)
    r = np.sqrt(-2.0 * np.log(u1))
    theta = 2.0 * math.pi * u2
    return r * np.cos(theta), r * np.sin(theta)


def sample_mos_variation(nl: Netlist, n_instances, vto_sigma=0.03, kp_rel_sigma=0.05,
                         base_seed=BASE_SEED, first_instance=0):
    """Per-instance MOSFET KP/VTO: VTO ~ N(card, vto_sigma), KP ~ N(card, kp_rel_sigma*card).

    Instance i uses PortableRNG(base_seed + i); each MOSFET (netlist order)
    draws one Box-Muller pair: the cosine sample perturbs VTO, the spare (sine)
    sample perturbs KP. Values are rounded to FP32.
    """
    seeds = np.arange(first_instance, first_instance + n_instances, dtype=np.uint64) + np.uint64(base_seed)
    rng = PCG32(seeds)
    n_mos = len(nl.mos)
    kp = np.empty((n_instances, n_mos), dtype=np.float32)
    vto = np.empty((n_instances, n_mos), dtype=np.float32)
    for j, m in enumerate(nl.mos):
        card = nl.models[m[6]]
        z_vto, z_kp = normal_pairs(rng)
        vto[:, j] = (card[3] + vto_sigma * z_vto).astype(np.float32)
        kp[:, j] = (card[2] * (1.0 + kp_rel_sigma * z_kp)).astype(np.float32)
    return kp, vto


@dataclass
class Instances:
    n: int
    mos_kp: np.ndarray | None = None
    mos_vto: np.ndarray | None = None
    vs_dc: np.ndarray | None = None

    def as_struct(self) -> A.KaramInstances:
        s = A.KaramInstances()
        s.n_instances = self.n
        self._kp = None if self.mos_kp is None else np.ascontiguousarray(self.mos_kp, dtype=np.float32)
        self._vto = None if self.mos_vto is None else np.ascontiguousarray(self.mos_vto, dtype=np.float32)
        self._vs = None if self.vs_dc is None else np.ascontiguousarray(self.vs_dc, dtype=np.float64)
        s.mos_kp = A.ptr(self._kp, C.c_float)
        s.mos_vto = A.ptr(self._vto, C.c_float)
        s.vs_dc = A.ptr(self._vs, C.c_double)
        return s

    def slice(self, i0, i1):
        g = lambda a: None if a is None else a[i0:i1]
        return Instances(i1 - i0, g(self.mos_kp), g(self.mos_vto), g(self.vs_dc))


def mc_instances(nl: Netlist, n_instances, **kw) -> Instances:
    kp, vto = sample_mos_variation(nl, n_instances, **kw)
    return Instances(n_instances, kp, vto)
