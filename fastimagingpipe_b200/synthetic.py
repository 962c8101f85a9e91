"""Seeded synthetic interferometer snapshots for the imaging + trigger path.

The reference is exercised on downloaded Measurement-Set snapshots
(README.md:38-41) that are not available here; these generators stand in for
them with the shapes, sizes and value distributions of the benchmark
configurations:

* antennas placed uniformly at random in a disk (optionally with a dense core),
  every pair i<j forming one baseline (128 antennas -> 8,128 baselines,
  512 -> 130,816);
* Earth-rotation uvw for snapshots a fixed number of seconds apart;
* point-source visibilities (lognormal fluxes, uniform positions inside the
  field of view) with an optional transient present in one snapshot only,
  plus complex Gaussian noise;
* the plane fit of each snapshot's uvw (FP64), giving the projected baseline
  matrix B and the 3x3 basis V that the reference's preprocessing produces
  (SVDPreprocessKernels.cu:41-206, SVD_MFS.py:38-110).

Everything is host-side numpy; nothing here runs on the GPU.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

C_LIGHT = 299792458.0
SIDEREAL_DAY_S = 86164.0905


@dataclasses.dataclass
class SnapshotSet:
    """Inputs of one FIpipe call, snapshot-concatenated like the reference's
    FITS inputs (pipe_interface.cpp:147-169): vis_re/vis_im [S*nb], B [S*nb*2]
    (row-major pairs), V [S*9] (row-major 3x3)."""

    vis_re: np.ndarray
    vis_im: np.ndarray
    B: np.ndarray
    V: np.ndarray
    num_baselines: int
    num_snapshots: int
    image_size: int
    cell_size: float
    unit_size: int
    frequency_hz: float
    uvw_m: Optional[np.ndarray] = None  # [S, nb, 3] metres (for plane-fit tests)
    transient_lm: Optional[tuple] = None
    flags: Optional[np.ndarray] = None  # [S, nb] bool, True = flagged

    def snapshot(self, k: int):
        nb = self.num_baselines
        return (self.vis_re[k * nb:(k + 1) * nb], self.vis_im[k * nb:(k + 1) * nb],
                self.B[k * nb * 2:(k + 1) * nb * 2], self.V[k * 9:(k + 1) * 9])


def antenna_layout(n_ant: int, radius_m: float, rng: np.random.Generator,
                   core_fraction: float = 0.0, core_radius_m: float = 0.0) -> np.ndarray:
    """ENU positions [n_ant, 3] (up = 0), uniform in a disk of `radius_m`;
    `core_fraction` of them uniform within `core_radius_m` instead."""
    n_core = int(round(n_ant * core_fraction))
    radii = np.empty(n_ant)
    radii[:n_core] = core_radius_m * np.sqrt(rng.random(n_core))
    radii[n_core:] = radius_m * np.sqrt(rng.random(n_ant - n_core))
    theta = 2.0 * np.pi * rng.random(n_ant)
    enu = np.zeros((n_ant, 3))
    enu[:, 0] = radii * np.cos(theta)
    enu[:, 1] = radii * np.sin(theta)
    return enu


def baseline_vectors(enu: np.ndarray) -> np.ndarray:
    """All pairs i<j (i outer), vector enu[j]-enu[i]: [n(n-1)/2, 3]."""
    i, j = np.triu_indices(enu.shape[0], k=1)
    return enu[j] - enu[i]


def enu_to_equatorial(b_enu: np.ndarray, lat_rad: float) -> np.ndarray:
    e, n, u = b_enu[:, 0], b_enu[:, 1], b_enu[:, 2]
    x = -math.sin(lat_rad) * n + math.cos(lat_rad) * u
    y = e
    z = math.cos(lat_rad) * n + math.sin(lat_rad) * u
    return np.stack([x, y, z], axis=1)


def uvw_from_xyz(xyz: np.ndarray, hour_angle_rad: float, dec_rad: float) -> np.ndarray:
    sh, ch = math.sin(hour_angle_rad), math.cos(hour_angle_rad)
    sd, cd = math.sin(dec_rad), math.cos(dec_rad)
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    u = sh * x + ch * y
    v = -sd * ch * x + sd * sh * y + cd * z
    w = cd * ch * x - cd * sh * y + sd * z
    return np.stack([u, v, w], axis=1)


def plane_fit(uvw_lambda: np.ndarray):
    """FP64 plane fit of one snapshot's uvw (in wavelengths): the top two
    principal axes of the centred coordinates (sign rule: the largest-magnitude
    component of each axis positive, SVDPreprocessKernels.cu:167-206), V row 2
    their cross product, and B the uncentred projection onto rows 0 and 1
    (SVD_MFS.py:105-110)."""
    x = np.asarray(uvw_lambda, dtype=np.float64)
    xc = x - x.mean(axis=0)
    cov = xc.T @ xc
    w, q = np.linalg.eigh(cov)  # ascending
    basis = np.stack([q[:, 2], q[:, 1]], axis=0)
    for c in range(2):
        a = int(np.argmax(np.abs(basis[c])))
        if basis[c, a] < 0:
            basis[c] = -basis[c]
    V = np.zeros((3, 3))
    V[:2] = basis
    V[2] = np.cross(V[0], V[1])
    B = x @ basis.T
    return B, V


def point_source_vis(uvw_lambda: np.ndarray, sources: np.ndarray) -> np.ndarray:
    """sum_s flux_s * exp(-2 pi i (u l + v m + w (n - 1))); sources [k, 3] =
    (l, m, flux)."""
    u, v, w = uvw_lambda[:, 0], uvw_lambda[:, 1], uvw_lambda[:, 2]
    out = np.zeros(u.shape[0], dtype=np.complex128)
    for l, m, s in sources:
        n = math.sqrt(max(0.0, 1.0 - l * l - m * m))
        out += s * np.exp(-2j * np.pi * (u * l + v * m + w * (n - 1.0)))
    return out


def make_snapshots(n_ant: int, radius_m: float, image_size: int, cell_size: float,
                   unit_size: int, *, n_snap: int = 3, freq_hz: float = 140e6,
                   core_fraction: float = 0.0, core_radius_m: float = 0.0,
                   n_sources: int = 20, transient_flux: float = 5.0,
                   transient_snapshot: Optional[int] = 1, noise_sigma: float = 0.1,
                   dec_deg: float = -30.0, lat_deg: float = -26.7,
                   hour_angle0_h: float = 1.5, dt_s: float = 10.0,
                   flag_fraction_max: float = 0.0, source_extent: float = 0.4,
                   flat_quadrant: bool = False, seed: int = 1) -> SnapshotSet:
    """Seeded snapshots of one beam.  Flagged baselines (up to
    `flag_fraction_max` of them, uniform per snapshot) are zero-padded the way
    the reference's preprocessing pads short snapshots
    (SVDPreprocessMain.cpp:264-291): vis 0 and B 0, still counted in nb."""
    rng = np.random.default_rng(seed)
    enu = antenna_layout(n_ant, radius_m, rng, core_fraction, core_radius_m)
    b_enu = baseline_vectors(enu)
    nb = b_enu.shape[0]
    xyz = enu_to_equatorial(b_enu, math.radians(lat_deg))
    fov = image_size * cell_size
    half = 0.5 * fov * source_extent
    lm = rng.uniform(-half, half, size=(n_sources, 2))
    if flat_quadrant:
        lm = np.abs(lm)  # every source in one quadrant: the rest of the sky is flat
    flux = rng.lognormal(mean=0.0, sigma=1.0, size=n_sources)
    sources = np.column_stack([lm, flux])
    t_lm = rng.uniform(-half, half, size=2)
    transient = np.array([[t_lm[0], t_lm[1], transient_flux]])

    lam = C_LIGHT / freq_hz
    vr = np.empty((n_snap, nb), np.float32)
    vi = np.empty((n_snap, nb), np.float32)
    Bs = np.empty((n_snap, nb, 2), np.float32)
    Vs = np.empty((n_snap, 3, 3), np.float32)
    uvw_all = np.empty((n_snap, nb, 3), np.float32)
    flags = np.zeros((n_snap, nb), bool)
    for k in range(n_snap):
        ha = 2.0 * np.pi * (hour_angle0_h * 3600.0 + k * dt_s) / SIDEREAL_DAY_S
        uvw = uvw_from_xyz(xyz, ha, math.radians(dec_deg))
        uvw_all[k] = uvw
        uvw_l = uvw / lam
        vis = point_source_vis(uvw_l, sources)
        if transient_snapshot is not None and k == transient_snapshot and transient_flux != 0:
            vis = vis + point_source_vis(uvw_l, transient)
        vis = vis + noise_sigma * (rng.standard_normal(nb) + 1j * rng.standard_normal(nb))
        B, V = plane_fit(uvw_l)
        if flag_fraction_max > 0:
            frac = rng.uniform(0.0, flag_fraction_max)
            flags[k] = rng.random(nb) < frac
            vis = np.where(flags[k], 0.0, vis)
            B = np.where(flags[k][:, None], 0.0, B)
        vr[k] = vis.real
        vi[k] = vis.imag
        Bs[k] = B
        Vs[k] = V
    return SnapshotSet(vis_re=vr.reshape(-1), vis_im=vi.reshape(-1), B=Bs.reshape(-1),
                       V=Vs.reshape(-1), num_baselines=nb, num_snapshots=n_snap,
                       image_size=image_size, cell_size=cell_size, unit_size=unit_size,
                       frequency_hz=freq_hz, uvw_m=uvw_all, transient_lm=tuple(t_lm),
                       flags=flags if flag_fraction_max > 0 else None)


# Benchmark configurations (the reference's headline shapes).

def config_small(seed: int = 1, **kw) -> SnapshotSet:
    """128 antennas in a 2 km disk (8,128 baselines), 3 snapshots 10 s apart at
    140 MHz, 20 sources + a 5 Jy transient in snapshot 2, noise 0.1; image
    512x512, cell 2.9e-5 rad, tile 16 (32x32 tLISI)."""
    args = dict(n_ant=128, radius_m=1000.0, image_size=512, cell_size=2.9e-5, unit_size=16)
    args.update(kw)
    return make_snapshots(seed=seed, **args)


def config_reference(seed: int = 1, **kw) -> SnapshotSet:
    """512 antennas in a 40 km layout with half of them within 1 km
    (130,816 baselines), 3 snapshots at 140 MHz, image 4096x4096,
    cell 7.2722e-6 rad, tile 32 (128x128 tLISI)."""
    args = dict(n_ant=512, radius_m=20000.0, core_fraction=0.5, core_radius_m=1000.0,
                image_size=4096, cell_size=7.2722e-6, unit_size=32)
    args.update(kw)
    return make_snapshots(seed=seed, **args)


def config_tiny(seed: int = 3, **kw) -> SnapshotSet:
    """A few-second oracle case: 48 antennas (1,128 baselines), image 128,
    tile 16."""
    args = dict(n_ant=48, radius_m=1000.0, image_size=128, cell_size=1.2e-4, unit_size=16)
    args.update(kw)
    return make_snapshots(seed=seed, **args)


@dataclasses.dataclass
class MfsSnapshot:
    """One multi-frequency snapshot: the unflagged samples of every baseline
    and channel (sample index = baseline + channel * baselines, the
    preprocessing's MFS order, SVDPreprocessMain.cpp:32-34), their projected
    coordinates B [nb, 2] and the plane basis V [3, 3]."""

    vis_re: np.ndarray
    vis_im: np.ndarray
    B: np.ndarray
    V: np.ndarray
    image_size: int
    cell_size: float
    unit_size: int

    @property
    def nb(self) -> int:
        return int(self.vis_re.shape[0])


def make_mfs_snapshots(n_ant: int, radius_m: float, image_size: int, cell_size: float,
                       unit_size: int, *, n_snap: int, freqs_hz, core_fraction: float = 0.0,
                       core_radius_m: float = 0.0, n_sources: int = 20,
                       transient_flux: float = 5.0, transient_snapshot: Optional[int] = None,
                       noise_sigma: float = 0.1, dec_deg: float = -30.0, lat_deg: float = -26.7,
                       hour_angle0_h: float = 1.5, dt_s: float = 10.0,
                       flag_fraction_max: float = 0.3, source_extent: float = 0.4,
                       seed: int = 1) -> list:
    """Seeded multi-channel snapshots with a uniform random 0..flag_fraction_max
    of their samples flagged and dropped (so nb differs between snapshots)."""
    rng = np.random.default_rng(seed)
    enu = antenna_layout(n_ant, radius_m, rng, core_fraction, core_radius_m)
    xyz = enu_to_equatorial(baseline_vectors(enu), math.radians(lat_deg))
    fov = image_size * cell_size
    half = 0.5 * fov * source_extent
    lm = rng.uniform(-half, half, size=(n_sources, 2))
    flux = rng.lognormal(mean=0.0, sigma=1.0, size=n_sources)
    sources = np.column_stack([lm, flux])
    t_lm = rng.uniform(-half, half, size=2)
    transient = np.array([[t_lm[0], t_lm[1], transient_flux]])
    out = []
    for k in range(n_snap):
        ha = 2.0 * np.pi * (hour_angle0_h * 3600.0 + k * dt_s) / SIDEREAL_DAY_S
        uvw = uvw_from_xyz(xyz, ha, math.radians(dec_deg))
        uvw_l = np.concatenate([uvw * (f / C_LIGHT) for f in freqs_hz])
        vis = point_source_vis(uvw_l, sources)
        if transient_snapshot is not None and k == transient_snapshot and transient_flux != 0:
            vis = vis + point_source_vis(uvw_l, transient)
        n = uvw_l.shape[0]
        vis = vis + noise_sigma * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
        B, V = plane_fit(uvw_l)
        keep = rng.random(n) >= rng.uniform(0.0, flag_fraction_max)
        out.append(MfsSnapshot(vis_re=np.ascontiguousarray(vis.real[keep], np.float32),
                               vis_im=np.ascontiguousarray(vis.imag[keep], np.float32),
                               B=np.ascontiguousarray(B[keep], np.float32).reshape(-1),
                               V=V.astype(np.float32).reshape(-1), image_size=image_size,
                               cell_size=cell_size, unit_size=unit_size))
    return out


def config_batching(image_size: int = 4096, n_snap: int = 8, n_chan: int = 8, seed: int = 1,
                    **kw) -> list:
    """The batching form's inputs for one image size: 512 antennas (40 km,
    half within 1 km), n_chan channels over 130-150 MHz, 0-30 % of each
    snapshot's samples flagged, tile 32, cell scaled so that the field of view
    is that of 4096 x 7.2722e-6 rad."""
    freqs = np.linspace(130e6, 150e6, n_chan)
    args = dict(n_ant=512, radius_m=20000.0, core_fraction=0.5, core_radius_m=1000.0,
                image_size=image_size, cell_size=7.2722e-6 * 4096 / image_size, unit_size=32,
                n_snap=n_snap, freqs_hz=freqs, flag_fraction_max=0.3)
    args.update(kw)
    return make_mfs_snapshots(seed=seed, **args)


@dataclasses.dataclass
class RawSnapshot:
    """One snapshot before preprocessing: baseline uvw in metres [rows, 3],
    channel frequencies [chans], and per sample (index row + chan * rows,
    SVDPreprocessMain.cpp:32-34) polarisations 0 and 3 (XX, YY) with flags and
    weights, as a Measurement Set holds them."""

    uvw_m: np.ndarray
    freqs_hz: np.ndarray
    xx: np.ndarray  # complex64 [rows * chans]
    yy: np.ndarray
    flag0: np.ndarray  # uint8
    flag3: np.ndarray
    weight0: np.ndarray  # float32
    weight3: np.ndarray
    image_size: int
    cell_size: float

    @property
    def num_samples(self) -> int:
        return int(self.xx.shape[0])


def make_raw_snapshot(n_ant: int = 64, radius_m: float = 1500.0, image_size: int = 256,
                      cell_size: float = 6e-5, freqs_hz=(130e6, 140e6, 150e6),
                      n_sources: int = 10, flag_fraction: float = 0.2,
                      pol_leak: float = 0.3, noise_sigma: float = 0.1,
                      dec_deg: float = -30.0, lat_deg: float = -26.7,
                      hour_angle_h: float = 1.5, seed: int = 7) -> RawSnapshot:
    """Seeded raw snapshot: Stokes I from point sources, XX = I + Q and
    YY = I - Q with a random Q of relative size `pol_leak`, independent noise
    per polarisation, each polarisation flagged with probability
    `flag_fraction` and weighted uniformly in [0.5, 1.5)."""
    rng = np.random.default_rng(seed)
    enu = antenna_layout(n_ant, radius_m, rng)
    xyz = enu_to_equatorial(baseline_vectors(enu), math.radians(lat_deg))
    ha = 2.0 * np.pi * hour_angle_h * 3600.0 / SIDEREAL_DAY_S
    uvw = uvw_from_xyz(xyz, ha, math.radians(dec_deg))
    fov = image_size * cell_size
    lm = rng.uniform(-0.2 * fov, 0.2 * fov, size=(n_sources, 2))
    flux = rng.lognormal(mean=0.0, sigma=1.0, size=n_sources)
    sources = np.column_stack([lm, flux])
    freqs = np.asarray(freqs_hz, np.float64)
    uvw_l = np.concatenate([uvw * (f / C_LIGHT) for f in freqs])  # row + chan * rows
    stokes_i = point_source_vis(uvw_l, sources)
    n = stokes_i.shape[0]
    q = pol_leak * np.abs(stokes_i) * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    noise = lambda: noise_sigma * (rng.standard_normal(n) + 1j * rng.standard_normal(n))
    xx = (stokes_i + q + noise()).astype(np.complex64)
    yy = (stokes_i - q + noise()).astype(np.complex64)
    flag0 = (rng.random(n) < flag_fraction).astype(np.uint8)
    flag3 = (rng.random(n) < flag_fraction).astype(np.uint8)
    w0 = rng.uniform(0.5, 1.5, n).astype(np.float32)
    w3 = rng.uniform(0.5, 1.5, n).astype(np.float32)
    return RawSnapshot(uvw_m=uvw.astype(np.float32), freqs_hz=freqs.astype(np.float32), xx=xx,
                       yy=yy, flag0=flag0, flag3=flag3, weight0=w0, weight3=w3,
                       image_size=image_size, cell_size=cell_size)
