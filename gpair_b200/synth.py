"""Seeded synthetic interferometric data sets (OIFITS tables) for the
reconstruction workloads.

The reference ships one OIFITS file and no generator; this module makes
OIFITS-like V2 and T3 tables with the shapes, sizes and noise of the
benchmark workloads:

* array: ``n_tel`` telescopes placed uniformly at random in a disk whose
  DIAMETER is ``array_diameter_m`` (all pairs are baselines);
* Earth-rotation synthesis at site latitude -24.6 deg, source declination
  -30 deg, ``n_ha`` hour angles evenly spaced over +-3 h, baselines rotated with
  the standard (u, v) projection of local (east, north, up) vectors;
* ``wavelengths`` spectral channels (one OI_WAVELENGTH table);
* V2 for every baseline, hour angle and channel; sigma(V2) = 0.01 + 0.05 V2;
* T3 for every triangle in ``triangles`` (all C(T,3) or the triangles that
  share telescope 0), closure-phase sigma 1 deg, amplitude sigma from the same
  model as V2;
* truth scenes are analytic (uniform / limb-darkened disks, elliptical
  Gaussians, points) so that no pixel grid is baked into the data. Positions
  are in mas from the image centre; the visibility convention matches the
  reference's DFT, exp(+2 pi i RPMAS u x) exp(-2 pi i RPMAS v y) with x, y the
  sky offsets (gpair1/trunk/gpair.c:242-243).

Scene and noise seeds are split so that the same scene can be re-observed
with fresh noise.
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np
from scipy import special

from .oifits import OIFits, T3Table, Vis2Table, WavelengthTable

RPMAS = (math.pi / 180.0) / 3600000.0  # radians per milliarcsecond
SITE_LAT_DEG = -24.6
DEC_DEG = -30.0


# ------------------------------------------------------------------ scenes

@dataclass
class Component:
    kind: str  # "disk", "lddisk", "gauss", "point"
    flux: float
    x: float = 0.0  # mas, from the image centre, +x as in the reference's DFT
    y: float = 0.0
    size: float = 0.0  # disk diameter or Gaussian major-axis FWHM, mas
    ratio: float = 1.0  # minor/major axis ratio (Gaussian)
    pa: float = 0.0  # position angle, radians
    ld: float = 0.0  # linear limb-darkening coefficient (lddisk)

    def vis(self, u: np.ndarray, v: np.ndarray) -> np.ndarray:
        """Complex visibility (flux-weighted) at u, v in wavelengths."""
        phase = np.exp(2j * np.pi * RPMAS * (u * self.x - v * self.y))
        if self.kind == "point":
            amp = np.ones_like(u)
        elif self.kind in ("disk", "lddisk"):
            rho = np.hypot(u, v)
            z = np.pi * self.size * RPMAS * rho
            zs = np.where(z == 0, 1.0, z)
            if self.kind == "disk":
                amp = np.where(z == 0, 1.0, 2.0 * special.j1(zs) / zs)
            else:
                a = self.ld
                num = (1 - a) * special.j1(zs) / zs + a * np.sqrt(np.pi / 2) * special.jv(1.5, zs) / zs ** 1.5
                amp = np.where(z == 0, 1.0, num / ((1 - a) / 2 + a / 3))
        elif self.kind == "gauss":
            c, s = math.cos(self.pa), math.sin(self.pa)
            up = c * u + s * v
            vp = -s * u + c * v
            fmaj = self.size * RPMAS
            fmin = self.size * self.ratio * RPMAS
            amp = np.exp(-(np.pi ** 2) / (4 * math.log(2)) * ((fmaj * up) ** 2 + (fmin * vp) ** 2))
        else:
            raise ValueError(self.kind)
        return self.flux * amp * phase


@dataclass
class Scene:
    components: List[Component] = field(default_factory=list)

    def vis(self, u, v):
        tot = sum(c.flux for c in self.components)
        acc = np.zeros(np.broadcast(u, v).shape, dtype=np.complex128)
        for c in self.components:
            acc += c.vis(u, v)
        return acc / tot


def scene_disk_spot(rng: np.random.Generator) -> Scene:
    """Uniform disk of 2 mas diameter plus a Gaussian spot (FWHM 0.5 mas, 20% flux) at a seeded offset."""
    r = rng.uniform(0.2, 0.8)
    t = rng.uniform(0, 2 * np.pi)
    return Scene([Component("disk", 0.8, size=2.0),
                  Component("gauss", 0.2, x=r * math.cos(t), y=r * math.sin(t), size=0.5)])


def scene_gaussians_points(rng: np.random.Generator, field_mas: float) -> Scene:
    """1-10 elliptical Gaussians plus 3 point sources inside the central part of the field."""
    comps = []
    ng = int(rng.integers(1, 11))
    half = 0.3 * field_mas
    for _ in range(ng):
        comps.append(Component("gauss", float(rng.uniform(0.2, 1.0)), x=float(rng.uniform(-half, half)),
                               y=float(rng.uniform(-half, half)), size=float(rng.uniform(0.05, 0.25) * field_mas),
                               ratio=float(rng.uniform(0.3, 1.0)), pa=float(rng.uniform(0, np.pi))))
    for _ in range(3):
        comps.append(Component("point", float(rng.uniform(0.05, 0.2)), x=float(rng.uniform(-half, half)),
                               y=float(rng.uniform(-half, half))))
    return Scene(comps)


def scene_stellar_surface(rng: np.random.Generator, diameter_mas: float = 15.0, n_spots: int = 50) -> Scene:
    """Limb-darkened disk with Gaussian spots of +-30% contrast."""
    comps = [Component("lddisk", 1.0, size=diameter_mas, ld=0.4)]
    R = diameter_mas / 2
    sb = 1.0 / (np.pi * R * R)  # mean surface brightness per mas^2
    for _ in range(n_spots):
        rr = R * math.sqrt(rng.uniform(0, 0.8))
        th = rng.uniform(0, 2 * np.pi)
        fw = rng.uniform(0.5, 2.0)
        area = np.pi / (4 * math.log(2)) * fw * fw
        comps.append(Component("gauss", float(rng.uniform(-0.3, 0.3) * sb * area), x=rr * math.cos(th),
                               y=rr * math.sin(th), size=fw))
    return Scene(comps)


# ----------------------------------------------------------------- arrays

def random_array(rng: np.random.Generator, n_tel: int, diameter_m: float) -> np.ndarray:
    """Telescope (east, north) positions uniform in a disk of the given diameter."""
    r = (diameter_m / 2) * np.sqrt(rng.uniform(0, 1, n_tel))
    t = rng.uniform(0, 2 * np.pi, n_tel)
    return np.stack([r * np.cos(t), r * np.sin(t)], axis=1)


def baseline_uv(enu: np.ndarray, ha_rad: np.ndarray, lat_deg=SITE_LAT_DEG, dec_deg=DEC_DEG):
    """(u, v) in metres of local baselines `enu` [...,2] (east, north; up = 0) at hour angles ha."""
    lat, dec = math.radians(lat_deg), math.radians(dec_deg)
    e, n = enu[..., 0], enu[..., 1]
    X = -math.sin(lat) * n
    Y = e
    Z = math.cos(lat) * n
    h = ha_rad
    u = np.sin(h) * X + np.cos(h) * Y
    v = -math.sin(dec) * np.cos(h) * X + math.sin(dec) * np.sin(h) * Y + math.cos(dec) * Z
    return u, v


@dataclass
class ArrayConfig:
    n_tel: int
    array_diameter_m: float
    n_ha: int
    wavelengths_m: Sequence[float]
    triangles: str = "all"  # "all" or "ref0" (triangles sharing telescope 0)
    bandwidth_m: float = 5e-8


def make_oifits(cfg: ArrayConfig, scene: Scene, array_seed: int, noise_seed: int,
                insname: str = "SYNTH", target_id: int = 1, t3amp_nan: bool = False) -> OIFits:
    """Observe `scene` with a seeded random array; returns OIFITS tables (one
    OI_WAVELENGTH, one OI_VIS2, one OI_T3 table)."""
    arng = np.random.default_rng(array_seed)
    nrng = np.random.default_rng(noise_seed)
    pos = random_array(arng, cfg.n_tel, cfg.array_diameter_m)
    ha = np.linspace(-3.0, 3.0, cfg.n_ha) * (np.pi / 12.0)
    lam = np.asarray(cfg.wavelengths_m, dtype=np.float32)
    nw = len(lam)
    lam64 = lam.astype(np.float64)
    pairs = list(itertools.combinations(range(cfg.n_tel), 2))
    if cfg.triangles == "ref0":
        tris = [(0, b, c) for b, c in itertools.combinations(range(1, cfg.n_tel), 2)]
    else:
        tris = list(itertools.combinations(range(cfg.n_tel), 3))

    def bl(a, b):
        return pos[b] - pos[a]

    # V2 rows: hour angle major, baseline minor
    vu, vv = [], []
    for h in ha:
        for a, b in pairs:
            u, v = baseline_uv(bl(a, b), h)
            vu.append(u)
            vv.append(v)
    vu = np.asarray(vu)
    vv = np.asarray(vv)
    V = scene.vis(vu[:, None] / lam64[None, :], vv[:, None] / lam64[None, :])
    v2 = np.abs(V) ** 2
    sig = 0.01 + 0.05 * v2
    v2obs = v2 + sig * nrng.standard_normal(v2.shape)
    nrec = len(vu)
    vis2 = Vis2Table(insname, np.full(nrec, target_id, np.int32), vu, vv, v2obs, sig,
                     np.zeros((nrec, nw), np.uint8))

    # T3 rows
    u1, v1, u2, v2c = [], [], [], []
    for h in ha:
        for a, b, c in tris:
            uu1, vv1 = baseline_uv(bl(a, b), h)
            uu2, vv2 = baseline_uv(bl(b, c), h)
            u1.append(uu1); v1.append(vv1); u2.append(uu2); v2c.append(vv2)
    u1, v1, u2, v2c = map(np.asarray, (u1, v1, u2, v2c))
    Vab = scene.vis(u1[:, None] / lam64, v1[:, None] / lam64)
    Vbc = scene.vis(u2[:, None] / lam64, v2c[:, None] / lam64)
    Vca = scene.vis(-(u1 + u2)[:, None] / lam64, -(v1 + v2c)[:, None] / lam64)
    T3 = Vab * Vbc * Vca
    amp = np.abs(T3)
    asig = 0.01 + 0.05 * amp
    phierr = np.ones_like(amp)
    phi = np.degrees(np.angle(T3)) + phierr * nrng.standard_normal(amp.shape)
    ampobs = amp + asig * nrng.standard_normal(amp.shape)
    if t3amp_nan:
        ampobs = np.full_like(ampobs, np.nan)
    nt = len(u1)
    t3 = T3Table(insname, np.full(nt, target_id, np.int32), u1, v1, u2, v2c, ampobs, asig, phi, phierr,
                 np.zeros((nt, nw), np.uint8))
    wave = WavelengthTable(insname, lam, np.full(nw, cfg.bandwidth_m, np.float32))
    return OIFits([wave], [vis2], [t3], target_id)


# ----------------------------------------------------------- workloads

@dataclass
class Workload:
    name: str
    image_width: int
    pixellation_mas: float
    array: ArrayConfig
    alpha: float
    scene_kind: str
    prior_flux: float = 1.0


def workload(name: str) -> Workload:
    """Named workloads: 'small' (64^2, 900 V2 / 600 T3), 'precision' (256^2, 21,120 V2 /
    70,400 T3), 'large' (1024^2, 194,560 V2 / 1,167,360 T3) and 'tiny' (a
    seconds-scale case for tests)."""
    if name == "small":
        return Workload(name, 64, 0.1, ArrayConfig(6, 330.0, 20, [1.5e-6, 1.65e-6, 1.8e-6], "ref0"),
                        1e-3, "disk_spot")
    if name == "precision":
        return Workload(name, 256, 0.05, ArrayConfig(12, 400.0, 40, list(np.linspace(1.45e-6, 1.85e-6, 8))),
                        1e-3, "gauss_points")
    if name == "large":
        return Workload(name, 1024, 0.02, ArrayConfig(20, 400.0, 64, list(np.linspace(1.45e-6, 1.85e-6, 16))),
                        1e-3, "stellar")
    if name == "tiny":
        return Workload(name, 32, 0.15, ArrayConfig(5, 200.0, 6, [1.6e-6, 1.7e-6], "all"), 1e-3, "disk_spot")
    raise KeyError(name)


def make_scene(kind: str, rng: np.random.Generator, field_mas: float) -> Scene:
    if kind == "disk_spot":
        return scene_disk_spot(rng)
    if kind == "gauss_points":
        return scene_gaussians_points(rng, field_mas)
    if kind == "stellar":
        return scene_stellar_surface(rng)
    raise KeyError(kind)


def make_workload_data(name: str, scene_seed: int = 1, noise_seed: int = 2, array_seed: int = 3) -> Tuple[Workload, OIFits]:
    w = workload(name)
    scene = make_scene(w.scene_kind, np.random.default_rng(scene_seed), w.image_width * w.pixellation_mas)
    return w, make_oifits(w.array, scene, array_seed, noise_seed)
