"""Synthetic granular media in the reference's data layout.

The reference builds media with its GEN_GRAIN command
(src/grain.f90:97-165 -> src/construct_grain.f90).  That setup is not on the
hot path; this module produces the same *kind* of arrays, in the same
conventions, so they can be handed to the GPU path (and to the CPU oracle in
the tests) exactly as the Fortran host would hand over its own arrays:

* grains are nodes: one grain per cell of an nx*ny grid, grain n (1-based)
  at cell (i, j) with n = i + nx*(j-1) (src/construct_grain.f90:160-189);
* grain2gridindex(0:N) / grain2grid(2, ncell) CSR, 1-based (data.f90:100-101);
* Hk magnitude hk(1,n) = |1 + k_sigma*N(0,1)| * Hk  ("k_sigma < 0" Gaussian,
  src/construct_grain.f90:1494-1506);
* easy axis uniform in cos(theta) inside a cone k_ang around +z with uniform
  azimuth (hk_uniform_p, :1672-1697; rotate, transform.f90:22-47);
* nearest-neighbour intralayer exchange CSR hxgrainindex(0:N), hxgrain(nnz)
  (1-based) and hx(nnz) in Oe, neighbours sorted by grain number
  (:1276-1317), with periodic wrap (iwrp, :1441-1455).  hx = L*ex/(Ms*A)
  (:1364); here the per-neighbour field `hex_oe` is given directly, i.e.
  ex = hex_oe*Ms*A/L.
* interlayer (vertical) exchange for columnar two-layer media: grain n of
  layer l couples to grain n of the adjacent layer with a field `hint_oe`
  (the reference's uhx/lhx CSR, :1006-1155).

Random draws use numpy's PCG64 (seeded), not the reference's MT streams: the
media are inputs, identical for the GPU path and the oracle.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np


@dataclasses.dataclass
class Layer:
    nx: int
    ny: int
    ms: np.ndarray            # (N,) emu/cc
    vol: np.ndarray           # (N,) cm^3
    axis: np.ndarray          # (N,3) unit easy axis
    hk: np.ndarray            # (N,2) Oe: Hk1, Hk2
    hk_scale: np.ndarray      # (N,)
    ms_scale: np.ndarray      # (N,)
    alpha_scale: np.ndarray   # (N,)
    alpha: float
    gamma: float
    floor_ms: float
    g2c_index: np.ndarray     # (N+1,) int32 cumulative (Fortran 0:N)
    g2c: np.ndarray           # (ncell,2) int32, 1-based (i,j)
    hx_index: Optional[np.ndarray]  # (N+1,) int32
    hx_grain: Optional[np.ndarray]  # (nnz,) int32 1-based
    hx: Optional[np.ndarray]        # (nnz,) Oe
    uhx: Optional[tuple] = None     # (index, grain, coef) coupling to layer l-1
    lhx: Optional[tuple] = None     # (index, grain, coef) coupling to layer l+1
    # schedule / thermal
    hdir: tuple = (0.0, 0.0, 1.0)
    t_start: float = -1e22
    t_end: float = 1e22
    s_start: float = 1.0
    s_end: float = 1.0
    scale: float = 1.0
    temperature: float = 0.0
    thermal: bool = False
    # time function of the uniform field (applied.f90:328-377): 0 = linear ramp,
    # 1 SIN, 2 COS, 3 EXP, 4 STE (trapezoidal square wave), 5 NEW
    func: int = 0
    amp: float = 0.0
    fgamma: float = 0.0
    phase: float = 0.0
    param: float = 0.0
    duty: float = 0.0
    moddepth: float = 0.0
    dc: float = 0.0
    # moving write head replacing the uniform field: dict(gap, z, hg, velocity,
    # x0, t0, bit_time, pattern, nbits) in cm, Oe, s (include/mrm_gpu.h
    # mrm_gpu_set_head_field)
    head: Optional[dict] = None
    # cubic anisotropy instead of uniaxial (field.f90:377-395): (N,3,3), row i
    # = crystal axis i of the grain in lab coordinates; hk holds K1, K2 as fields
    cubic_axis: Optional[np.ndarray] = None
    # tabulated (moving) field profile replacing the uniform direction, scaled by
    # the layer's time scale: dict(xpos, ypos, vfld (ny_tab, nx_tab, 3), vel,
    # offset, ref, t_origin) (include/mrm_gpu.h mrm_gpu_set_field_table)
    field_table: Optional[dict] = None
    # LLB integrator (llgp%llb): dict(spin, tc (N,) K, lambda_ms (N,) Oe)
    # (include/mrm_gpu.h mrm_gpu_set_llb)
    llb: Optional[dict] = None
    # MT integrator (llgp%mt): dict(spin, lambda_ms (N,) Oe, meq_bs, garanin_tau)
    # (include/mrm_gpu.h mrm_gpu_set_mt)
    mt: Optional[dict] = None
    # moving super-Gaussian temperature profile: dict of GpuSim.set_temp_profile's
    # arguments (include/mrm_gpu.h mrm_gpu_set_temp_profile)
    temp_profile: Optional[dict] = None
    # Zhang integrator (llgp%zhang): dict(spin, lambda_ms, meq_bs, garanin_tau)
    zhang: Optional[dict] = None
    # temperature scaling of Ms, alpha, Hk: dict of GpuSim.set_temp_scaling's
    # arguments (tc, msexp, hkexp, use_mag, tables) (include/mrm_gpu.h
    # mrm_gpu_set_temp_scaling); the layer's scales are then uploaded as 1
    temp_scaling: Optional[dict] = None

    @property
    def N(self) -> int:
        return int(self.ms.shape[0])


@dataclasses.dataclass
class Medium:
    nx: int
    ny: int
    dx: float
    dy: float
    dz: List[float]
    il_space: List[float]
    layers: List[Layer]
    boundary: int = 1          # 0 periodic (reference), 1 open / zero-padded 2x
    images: int = 2
    # moving demag window: dict(nx, ny, v=(vx, vy), offset=(ox, oy)) (include/mrm_gpu.h
    # mrm_gpu_set_window); None: the demag covers the whole grid
    window: Optional[dict] = None
    space_to_sul: float = 0.0
    sul_mu: float = 1.0
    head_mu: float = 1.0
    fly_height: float = 0.0
    m0: Optional[List[np.ndarray]] = None   # initial m per layer (N,3)

    @property
    def n_lay(self) -> int:
        return len(self.layers)

    @property
    def n_grains(self) -> int:
        return sum(l.N for l in self.layers)


def lattice_maps(nx: int, ny: int):
    """grains-as-nodes grain<->cell CSR (construct_grain.f90:182-189)."""
    n = nx * ny
    idx = np.arange(n + 1, dtype=np.int32)
    jj, ii = np.divmod(np.arange(n), nx)
    g2c = np.stack([ii + 1, jj + 1], axis=1).astype(np.int32)
    return idx, g2c


def lattice_exchange(nx: int, ny: int, hex_oe):
    """4-neighbour periodic exchange CSR, neighbours sorted by grain number.

    hex_oe: scalar or (N,) per-grain field per unit shared edge fraction.
    Shared edges that wrap onto the same neighbour twice accumulate
    (construct_grain.f90:1298-1316).
    """
    n = nx * ny
    hexa = np.broadcast_to(np.asarray(hex_oe, dtype=np.float64), (n,))
    index = np.zeros(n + 1, dtype=np.int32)
    grains: list = []
    coefs: list = []
    if nx >= 3 and ny >= 3:
        g = np.arange(n)
        j, i = np.divmod(g, nx)
        nb = np.stack([
            i + nx * ((j - 1) % ny),        # (i, j-1)   shared length dx
            (i - 1) % nx + nx * j,          # (i-1, j)   shared length dy
            (i + 1) % nx + nx * j,          # (i+1, j)   shared length dy
            i + nx * ((j + 1) % ny),        # (i, j+1)   shared length dx
        ], axis=1)
        order = np.argsort(nb, axis=1, kind="stable")
        nbs = np.take_along_axis(nb, order, axis=1)
        index[1:] = 4 * np.arange(1, n + 1)
        hx_grain = (nbs + 1).astype(np.int32).reshape(-1)
        hx = np.repeat(hexa, 4)
        return index, hx_grain, hx.astype(np.float64)
    for g in range(n):
        j, i = divmod(g, nx)
        acc = {}
        for nbg in (i + nx * ((j - 1) % ny), (i - 1) % nx + nx * j,
                    (i + 1) % nx + nx * j, i + nx * ((j + 1) % ny)):
            if nbg != g:
                acc[nbg] = acc.get(nbg, 0.0) + 1.0
        for k in sorted(acc):
            grains.append(k + 1)
            coefs.append(acc[k] * hexa[g])
        index[g + 1] = len(grains)
    return index, np.asarray(grains, np.int32), np.asarray(coefs, np.float64)


def easy_axes(rng: np.random.Generator, n: int, k_ang_deg: float) -> np.ndarray:
    """uniform-in-cos(theta) cone around +z, uniform azimuth (construct_grain.f90:1672-1697)."""
    tsig = abs(k_ang_deg) * math.pi / 180.0
    phi = 2.0 * math.pi * rng.random(n)
    if tsig == 0.0:
        theta = np.zeros(n)
    else:
        u = rng.random(n)
        theta = np.arccos(np.minimum(1.0, np.maximum(math.cos(tsig), 1.0 - u * (1.0 - math.cos(tsig)))))
    # rotate(phi_n=0, theta_n=0, phi, theta) (transform.f90:22-47)
    st = np.sin(theta)
    return np.stack([np.cos(phi) * st, np.sin(phi) * st, np.cos(theta)], axis=1)


def hk_magnitudes(rng: np.random.Generator, n: int, hk: float, k_sigma: float) -> np.ndarray:
    """|1 + k_sigma*N(0,1)| * hk for k_sigma<0 (Gaussian), exp(k_sigma*N) for k_sigma>0."""
    x = 1.0 + abs(k_sigma) * rng.standard_normal(n)
    if k_sigma > 0:
        x = np.exp(x - 1.0)
    return np.abs(x) * hk


def make_layer(rng, nx, ny, dx, dy, dz, ms, hk, k_sigma, k_ang_deg, hex_oe, alpha,
               gamma=1.76e7, hk2=0.0) -> Layer:
    n = nx * ny
    g2c_index, g2c = lattice_maps(nx, ny)
    hkm = hk_magnitudes(rng, n, hk, k_sigma)
    hkarr = np.stack([hkm, np.full(n, 0.0) + hk2 * hkm / max(hk, 1e-300)], axis=1)
    axis = easy_axes(rng, n, k_ang_deg)
    if hex_oe != 0.0:
        hx_index, hx_grain, hx = lattice_exchange(nx, ny, hex_oe)
    else:
        hx_index = hx_grain = hx = None
    return Layer(
        nx=nx, ny=ny,
        ms=np.full(n, float(ms)), vol=np.full(n, dx * dy * dz),
        axis=axis, hk=hkarr,
        hk_scale=np.ones(n), ms_scale=np.ones(n), alpha_scale=np.ones(n),
        alpha=float(alpha), gamma=float(gamma), floor_ms=0.01,
        g2c_index=g2c_index, g2c=g2c,
        hx_index=hx_index, hx_grain=hx_grain, hx=hx,
    )


def cubic_frames(rng: np.random.Generator, n: int) -> np.ndarray:
    """(n,3,3) uniformly random orthonormal crystal frames (rows = axes)."""
    q, r = np.linalg.qr(rng.standard_normal((n, 3, 3)))
    q *= np.sign(np.diagonal(r, axis1=1, axis2=2))[:, None, :]
    return np.ascontiguousarray(np.transpose(q, (0, 2, 1)))


def cubic_medium(side: int, *, k1_oe: float = 4000.0, k2_oe: float = 1000.0, seed: int = 1,
                 temperature: float = 0.0, boundary: int = 1, hex_oe: float = 500.0) -> Medium:
    """M(H) medium of the 4,096/65,536-grain kind with cubic anisotropy:
    random crystal frames per grain, K1 and K2 as fields (hk(1), hk(2))."""
    med = mh_medium(side, temperature=temperature, boundary=boundary, seed=seed, hex_oe=hex_oe)
    lay = med.layers[0]
    rng = np.random.default_rng(seed + 1000)
    lay.cubic_axis = cubic_frames(rng, lay.N)
    lay.hk = np.stack([np.full(lay.N, k1_oe), np.full(lay.N, k2_oe)], axis=1)
    return med


def grain_map_medium(nx: int = 16, ny: int = 16, *, seed: int = 1, temperature: float = 0.0,
                     empty_frac: float = 0.05, hex_oe: float = 300.0, boundary: int = 1, ms: float = 700.0,
                     hk: float = 15000.0, pitch_nm: float = 8.0, thickness_nm: float = 10.0) -> Medium:
    """M(H) medium whose grains cover one to four cells (1x1, 2x1, 1x2, 2x2
    blocks, clipped where cells are taken) with a few empty cells: the
    grain <-> cell maps of get_mag / get_magnetostatic (data.f90:322-390,
    field.f90:438-517).  Exchange between grains sharing a cell edge."""
    rng = np.random.default_rng(seed)
    owner = -np.ones((ny, nx), dtype=np.int64)
    grains = []
    shapes = [(1, 1), (2, 1), (1, 2), (2, 2)]
    for j in range(ny):
        for i in range(nx):
            if owner[j, i] >= 0 or rng.random() < empty_frac:
                continue
            w, h = shapes[int(rng.integers(0, len(shapes)))]
            cells = [(i + a, j + b) for b in range(h) for a in range(w)
                     if i + a < nx and j + b < ny and owner[j + b, i + a] < 0]
            for ci, cj in cells:
                owner[cj, ci] = len(grains)
            grains.append(cells)
    n = len(grains)
    g2c_index = np.concatenate([[0], np.cumsum([len(c) for c in grains])]).astype(np.int32)
    g2c = np.array([(ci + 1, cj + 1) for c in grains for ci, cj in c], dtype=np.int32)
    nbrs = []
    for g, cells in enumerate(grains):
        s_ = set()
        for ci, cj in cells:
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                a, b = ci + di, cj + dj
                if 0 <= a < nx and 0 <= b < ny and owner[b, a] >= 0 and owner[b, a] != g:
                    s_.add(int(owner[b, a]))
        nbrs.append(sorted(s_))
    hx_index = np.concatenate([[0], np.cumsum([len(x) for x in nbrs])]).astype(np.int32)
    hx_grain = np.array([q + 1 for x in nbrs for q in x], dtype=np.int32)
    hx = np.full(len(hx_grain), float(hex_oe))
    dx = dy = pitch_nm * 1e-7
    dz = thickness_nm * 1e-7
    ncell = np.array([len(c) for c in grains], dtype=float)
    lay = Layer(nx=nx, ny=ny, ms=np.full(n, float(ms)), vol=ncell * dx * dy * dz,
                axis=easy_axes(rng, n, 3.0), hk=np.stack([hk_magnitudes(rng, n, hk, -0.05), np.zeros(n)], axis=1),
                hk_scale=np.ones(n), ms_scale=np.ones(n), alpha_scale=np.ones(n), alpha=0.1, gamma=1.76e7,
                floor_ms=0.01, g2c_index=g2c_index, g2c=g2c, hx_index=hx_index, hx_grain=hx_grain, hx=hx)
    a = math.radians(10.0)
    lay.hdir = (math.sin(a), 0.0, math.cos(a))
    lay.t_start, lay.t_end, lay.s_start, lay.s_end, lay.scale = 0.0, 2e-10, 20000.0, -20000.0, 1.0
    lay.temperature = float(temperature)
    lay.thermal = temperature > 0.0
    m0 = np.zeros((n, 3))
    m0[:, 2] = 1.0
    return Medium(nx=nx, ny=ny, dx=dx, dy=dy, dz=[dz], il_space=[0.0], layers=[lay], boundary=boundary, m0=[m0])


def columnar_coupling(n: int, coef_oe: float):
    idx = np.arange(n + 1, dtype=np.int32)
    grain = np.arange(1, n + 1, dtype=np.int32)
    return idx, grain, np.full(n, float(coef_oe))


def mh_medium(side: int, *, pitch_nm: float = 8.0, thickness_nm: float = 10.0, ms: float = 700.0,
              hk: float = 15000.0, k_sigma: float = -0.05, k_ang_deg: float = 3.0,
              hex_oe: float = 500.0, alpha: float = 0.1, h_max: float = 20000.0,
              angle_deg: float = 10.0, ramp_s: float = 2e-9, temperature: float = 0.0,
              boundary: int = 1, seed: int = 1, ny: Optional[int] = None) -> Medium:
    """Single-layer M(H) medium (the 4,096- and 65,536-grain workloads).

    Uniform field along (sin a, 0, cos a) ramped linearly from +h_max to
    -h_max over ramp_s (applied.f90:871-883); m starts along +z.
    """
    nx = side
    ny = side if ny is None else ny
    rng = np.random.default_rng(seed)
    dx = dy = pitch_nm * 1e-7
    dz = thickness_nm * 1e-7
    lay = make_layer(rng, nx, ny, dx, dy, dz, ms, hk, k_sigma, k_ang_deg, hex_oe, alpha)
    a = math.radians(angle_deg)
    lay.hdir = (math.sin(a), 0.0, math.cos(a))
    lay.t_start, lay.t_end, lay.s_start, lay.s_end, lay.scale = 0.0, ramp_s, h_max, -h_max, 1.0
    lay.temperature = float(temperature)
    lay.thermal = temperature > 0.0
    m0 = np.zeros((lay.N, 3))
    m0[:, 2] = 1.0
    return Medium(nx=nx, ny=ny, dx=dx, dy=dy, dz=[dz], il_space=[0.0], layers=[lay],
                  boundary=boundary, m0=[m0])


def two_layer_medium(nx: int = 1024, ny: int = 256, *, pitch_nm: float = 7.0, seed: int = 1,
                     temperature: float = 300.0, hint_oe: float = 2000.0, hex_oe: float = 500.0,
                     alpha: float = 0.1, boundary: int = 1) -> Medium:
    """Exchange-coupled hard/soft recording bilayer (the two-layer write workload)."""
    rng = np.random.default_rng(seed)
    dx = dy = pitch_nm * 1e-7
    hard = make_layer(rng, nx, ny, dx, dy, 8e-7, 800.0, 18000.0, -0.05, 3.0, hex_oe, alpha)
    soft = make_layer(rng, nx, ny, dx, dy, 4e-7, 900.0, 6000.0, -0.05, 3.0, hex_oe, alpha)
    n = nx * ny
    # layer 1 is the top layer (nearest the head), layer 2 below it (tensor.f90:149-200)
    hard.lhx = columnar_coupling(n, hint_oe)
    soft.uhx = columnar_coupling(n, hint_oe)
    for lay in (hard, soft):
        lay.temperature = float(temperature)
        lay.thermal = temperature > 0.0
    m0 = [np.tile([0.0, 0.0, 1.0], (n, 1)), np.tile([0.0, 0.0, 1.0], (n, 1))]
    return Medium(nx=nx, ny=ny, dx=dx, dy=dy, dz=[8e-7, 4e-7], il_space=[0.0, 0.0],
                  layers=[hard, soft], boundary=boundary, m0=m0)


def prbs_pattern(nbits: int = 64, seed: int = 1) -> int:
    """Seeded pseudo-random bit pattern: the PRBS7 sequence (x^7 + x^6 + 1
    linear-feedback shift register) started from a seed-dependent non-zero
    state; bit k of the result is the k-th bit written."""
    state = (seed * 0x5B + 0x2D) & 0x7F or 1
    out = 0
    for k in range(nbits):
        bit = ((state >> 6) ^ (state >> 5)) & 1
        state = ((state << 1) | bit) & 0x7F
        out |= (state & 1) << k
    return out


def karlqvist_deep_gap(peak_oe: float, gap_cm: float, z_cm: float) -> float:
    """Deep-gap field whose Karlqvist h_x peak (under the gap centre) at
    distance z equals peak_oe: h_x(0, z) = 2 Hg/pi atan(gap / (2 z))."""
    return peak_oe * math.pi / (2.0 * math.atan(gap_cm / (2.0 * z_cm)))


def head_write_medium(nx: int = 1024, ny: int = 256, *, seed: int = 1, prbs_seed: int = 1,
                      temperature: float = 300.0, gap_nm: float = 25.0, fly_nm: float = 6.0,
                      peak_oe: float = 12000.0, velocity_cm_s: float = 2000.0, bit_nm: float = 15.0,
                      nbits: int = 64, boundary: int = 1) -> Medium:
    """Two-layer recording write (the 1,024 x 256 x 2-layer workload): the
    hard/soft bilayer of two_layer_medium written by a Karlqvist ring head
    (gap 25 nm, 6 nm above the top layer, 12 kOe peak at the top surface)
    moving down-track at 20 m/s, polarity from a seeded 64-bit PRBS at 15 nm
    bit length (bit time = bit length / velocity).  The head enters at the
    left edge of the grid at t = 0.  Layer 0 is the top layer."""
    med = two_layer_medium(nx, ny, seed=seed, temperature=temperature, boundary=boundary)
    gap, fly = gap_nm * 1e-7, fly_nm * 1e-7
    hg = karlqvist_deep_gap(peak_oe, gap, fly)
    pattern = prbs_pattern(nbits, prbs_seed)
    depth = 0.0
    for l, lay in enumerate(med.layers):
        z = fly + depth + 0.5 * med.dz[l]
        depth += med.dz[l] + med.il_space[l]
        lay.head = dict(gap=gap, z=z, hg=hg, velocity=velocity_cm_s, x0=0.0, t0=0.0,
                        bit_time=bit_nm * 1e-7 / velocity_cm_s, pattern=pattern, nbits=nbits)
    return med


def tabulated_head_profile(gap: float, z: float, hg: float, track_width: float, *, nx_tab: int = 97,
                           ny_tab: int = 33, x_half: Optional[float] = None, y_half: Optional[float] = None):
    """A write-head field table (the stand-in for a FEM head-field file): the
    Karlqvist field of a ring head of gap `gap` at distance z, deep-gap field hg,
    times a cross-track envelope 0.5 (tanh((y + w/2)/e) - tanh((y - w/2)/e)),
    e = gap/4, on nodes that crowd towards the gap (x) and the track centre (y).
    Returns (xpos, ypos, vfld (ny_tab, nx_tab, 3)) in cm and Oe."""
    xh = 8.0 * gap if x_half is None else x_half
    yh = track_width if y_half is None else y_half
    u = np.linspace(-1.0, 1.0, nx_tab)
    xpos = xh * np.sinh(2.0 * u) / np.sinh(2.0)
    ypos = yh * np.sinh(1.5 * np.linspace(-1.0, 1.0, ny_tab)) / np.sinh(1.5)
    a, b = xpos + 0.5 * gap, xpos - 0.5 * gap
    kx = hg / np.pi * (np.arctan(a / z) - np.arctan(b / z))
    kz = hg / (2.0 * np.pi) * np.log((b * b + z * z) / (a * a + z * z))
    e = 0.25 * gap
    env = 0.5 * (np.tanh((ypos + 0.5 * track_width) / e) - np.tanh((ypos - 0.5 * track_width) / e))
    vfld = np.zeros((ny_tab, nx_tab, 3))
    vfld[..., 0] = env[:, None] * kx[None, :]
    vfld[..., 2] = env[:, None] * kz[None, :]
    return xpos, ypos, vfld


def table_write_medium(nx: int = 1024, ny: int = 256, *, seed: int = 1, temperature: float = 300.0,
                       gap_nm: float = 25.0, fly_nm: float = 6.0, peak_oe: float = 12000.0,
                       velocity_cm_s: float = 2000.0, bit_nm: float = 15.0, track_nm: Optional[float] = None,
                       rise_frac: float = 0.2, boundary: int = 1) -> Medium:
    """The two-layer write of head_write_medium driven the way the reference
    drives writes: a tabulated head-field profile per layer (tabulated_head_profile
    at the layer's depth, track width 3/4 of the grid's width by default) moving
    down-track at `velocity_cm_s` from the grid's left edge at t = 0, centred
    cross-track, its polarity from the STE time function (square wave of
    period two bit times, rise time rise_frac of a bit), i.e. alternating bits."""
    med = two_layer_medium(nx, ny, seed=seed, temperature=temperature, boundary=boundary)
    gap, fly = gap_nm * 1e-7, fly_nm * 1e-7
    hg = karlqvist_deep_gap(peak_oe, gap, fly)
    tw = 0.75 * ny * med.dy if track_nm is None else track_nm * 1e-7
    tbit = bit_nm * 1e-7 / velocity_cm_s
    depth = 0.0
    for l, lay in enumerate(med.layers):
        z = fly + depth + 0.5 * med.dz[l]
        depth += med.dz[l] + med.il_space[l]
        xpos, ypos, vfld = tabulated_head_profile(gap, z, hg, tw)
        lay.field_table = dict(xpos=xpos, ypos=ypos, vfld=vfld, vel=(velocity_cm_s, 0.0), offset=(0.0, None),
                               ref=(0.0, 0.0), t_origin=0.0)
        lay.func, lay.amp, lay.fgamma, lay.param, lay.dc, lay.scale = 4, 1.0, 2.0 * tbit, rise_frac * tbit, 0.0, 1.0
        lay.phase, lay.duty, lay.moddepth = 0.0, 0.0, 0.0
    return med


def llb_medium(side: int = 32, *, temperature: float = 600.0, tc: float = 700.0, tc_sigma: float = 0.03,
               spin: float = 0.5, seed: int = 1, boundary: int = 1, h_oe: float = 8000.0) -> Medium:
    """A heat-assisted write of a single FePt-like layer with the LLB integrator:
    the M(H) medium of mh_medium at a uniform temperature below a grain-to-grain
    distributed Curie temperature (Tc ~ N(tc, tc_sigma tc)), spin S, and the
    mean-field coupling of each grain's Tc, lambdaMs = 3 Tc / ((g mu_B/k_B)
    (S + 1)) (the mean-field Tc of push_llb's Langevin form, lambda_m =
    lambdaMs (S+1)/S, is (g mu_B/k_B) S lambda_m / 3), under a constant
    reversing field of h_oe along the medium's field direction; the anisotropy
    and Ms scales stay the inputs (no temperature scaling unless the layer's
    temp_scaling is set)."""
    med = mh_medium(side, seed=seed, boundary=boundary, temperature=temperature)
    rng = np.random.default_rng(seed + 1000)
    for lay in med.layers:
        lay.thermal = True
        lay.temperature = temperature
        lay.t_start, lay.t_end = -1e22, 1e22
        lay.s_start = lay.s_end = 1.0
        lay.scale = -h_oe
        tcs = np.clip(rng.normal(tc, tc_sigma * tc, lay.N), temperature * 1.02, None)
        lay.llb = dict(spin=spin, tc=tcs, lambda_ms=3.0 * tcs / (1.343427768e-4 * (spin + 1.0)))
    return med


def mt_medium(side: int = 32, *, meq_bs: bool = False, garanin_tau: bool = False, **kw) -> Medium:
    """llb_medium's heat-assisted layer driven by the MT integrator instead:
    the same spin and mean-field coupling (lambdaMs from each grain's Tc, as
    the Brillouin (meq_bs) or Langevin mean field of push_mt fixes Tc)."""
    med = llb_medium(side, **kw)
    for lay in med.layers:
        lb = lay.llb
        sp = lb["spin"]
        # mean-field Tc: B_S'(0) = (S+1)/(3S), so lambdaMs = 3 Tc/((g mu_B/k_B)(S+1))
        # for B_S; the Langevin form takes the same lambdaMs through lambda_m (S+1)/S
        lay.mt = dict(spin=sp, lambda_ms=lb["lambda_ms"], meq_bs=meq_bs, garanin_tau=garanin_tau)
        lay.llb = None
    return med


def hamr_medium(side: int = 64, *, seed: int = 1, background: float = 300.0, peak: float = 450.0,
                sigma_nm: float = 60.0, velocity_cm_s: float = 2000.0, **kw) -> Medium:
    """A heat-assisted write: llb_medium's layer at a background temperature with
    a laser spot (second-order super-Gaussian, 1/e half width sigma_nm, peak
    rise `peak` above the background) moving down-track from the grid's left
    edge at `velocity_cm_s`, under the medium's reversing field."""
    med = llb_medium(side, seed=seed, temperature=background, **kw)
    for lay in med.layers:
        lay.temperature = background
        lay.temp_profile = dict(background=background, dtemp=peak, sigma=(sigma_nm * 1e-7, sigma_nm * 1e-7), expn=1,
                                vel=(velocity_cm_s, 0.0), offset=(0.0, None), ref=(0.0, 0.0), t_origin=0.0)
    return med


def zhang_medium(side: int = 32, *, meq_bs: bool = False, garanin_tau: bool = False, **kw) -> Medium:
    """mt_medium's heat-assisted layer driven by the Zhang integrator."""
    med = mt_medium(side, meq_bs=meq_bs, garanin_tau=garanin_tau, **kw)
    for lay in med.layers:
        lay.zhang, lay.mt = lay.mt, None
    return med
