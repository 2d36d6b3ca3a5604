"""In-memory magnetostatic model passed across the C-ABI.

Mirrors the reference's ``NonlinearModel`` (gpu_solver/src/physics/nonlinear_model.h:83-100):
nodes in metres, P1 triangles with one material label each, materials carrying the
reluctivity law, coil current density per amp, permanent-magnet coercivity and angle,
raw B-H curves (the library builds FEMM's DC spline from them), homogeneous or
prescribed Dirichlet nodes, signed periodic/anti-periodic node pairs, the circuit
count and the planar depth.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

MU0 = 4.0e-7 * np.pi

PLANAR = 0
AXISYMMETRIC = 1


@dataclass
class AirGap:
    """FEMM's native air-gap element (fg_air_gap_element): an untriangulated annular band.
    nodes / weights [points, 4]: per band point the inner-ring nodes n0, n1 bracketing it
    and the outer-ring ones n2, n3, each weight the +1 / -1 sign of the ring copy;
    inner_shift / outer_shift place each ring's first node in units of one arc."""
    nodes: np.ndarray
    weights: np.ndarray
    inner_radius_m: float
    outer_radius_m: float
    arc_length_deg: float
    inner_shift: float = 0.0
    outer_shift: float = 0.0
    antiperiodic: bool = False
    center_m: Tuple[float, float] = (0.0, 0.0)

    def __post_init__(self):
        self.nodes = np.ascontiguousarray(self.nodes, dtype=np.int32).reshape(-1, 4)
        self.weights = np.ascontiguousarray(self.weights, dtype=np.float64).reshape(-1, 4)


@dataclass
class Model:
    xy: np.ndarray  # [N, 2] float64, metres (x, y) or (r, z)
    tri: np.ndarray  # [E, 3] int32, CCW
    tri_mat: np.ndarray  # [E] int32
    nu0: np.ndarray  # [M] float64, 1 / (mu0 mu_r)
    alpha: np.ndarray  # [M] float64
    j_per_a: np.ndarray  # [M] float64, A/m^2 per circuit amp
    hc: np.ndarray  # [M] float64, A/m
    mag_deg: np.ndarray  # [M] float64
    curve_index: np.ndarray  # [M] int32, -1 = linear material
    circuit_index: np.ndarray  # [M] int32, -1 = not driven
    group: np.ndarray  # [M] int32
    curves: List[Tuple[np.ndarray, np.ndarray]]  # raw (B [T], H [A/m]) points, origin first
    dir_nodes: np.ndarray  # [D] int32
    dir_values: np.ndarray  # [D] float64
    con_a: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    con_b: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    con_sign: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int8))
    circuit_count: int = 1
    depth_m: float = 1.0
    problem_type: int = PLANAR
    name: str = "model"
    ages: List[AirGap] = field(default_factory=list)

    def __post_init__(self):
        self.xy = np.ascontiguousarray(self.xy, dtype=np.float64).reshape(-1, 2)
        self.tri = np.ascontiguousarray(self.tri, dtype=np.int32).reshape(-1, 3)
        self.tri_mat = np.ascontiguousarray(self.tri_mat, dtype=np.int32)
        for name in ("nu0", "alpha", "j_per_a", "hc", "mag_deg", "dir_values"):
            setattr(self, name, np.ascontiguousarray(getattr(self, name), dtype=np.float64))
        for name in ("curve_index", "circuit_index", "group", "dir_nodes", "con_a", "con_b"):
            setattr(self, name, np.ascontiguousarray(getattr(self, name), dtype=np.int32))
        self.con_sign = np.ascontiguousarray(self.con_sign, dtype=np.int8)
        self.curves = [
            (np.ascontiguousarray(b, dtype=np.float64), np.ascontiguousarray(h, dtype=np.float64))
            for b, h in self.curves
        ]

    @property
    def node_count(self) -> int:
        return int(self.xy.shape[0])

    @property
    def tri_count(self) -> int:
        return int(self.tri.shape[0])

    @property
    def mat_count(self) -> int:
        return int(self.nu0.shape[0])

    def curve_arrays(self):
        """Concatenated raw curve points and their offsets ([curves + 1])."""
        offsets = [0]
        for b, _ in self.curves:
            offsets.append(offsets[-1] + len(b))
        cb = np.concatenate([b for b, _ in self.curves]) if self.curves else np.zeros(1)
        ch = np.concatenate([h for _, h in self.curves]) if self.curves else np.zeros(1)
        return (np.asarray(offsets, dtype=np.int32), np.ascontiguousarray(cb, dtype=np.float64),
                np.ascontiguousarray(ch, dtype=np.float64))
