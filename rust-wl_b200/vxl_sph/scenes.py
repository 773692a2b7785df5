"""Seeded synthetic WCSPH scenes (dam breaks in Akinci-walled tanks).

The reference has no stored scenes; its benchmarks build lattice blocks on the fly
(crates/vxl-phys-fluid/examples/sph_scale.rs:27-36) and tanks of static boxes
(crates/vxl-phys-gpu/examples/gpu_tick_probe.rs:20-63). These builders make the same
kinds of scenes at the workload sizes this library is measured on:

  dam0   16,384 fluid particles (16 x 32 x 32) at s = 0.02 in a 1.0 x 0.64 x 0.64 m tank
  dam1   1,000,000 (100^3) at s = 0.01 in a 2 x 2 x 1 m tank (fill 25% by volume)
  dam10m 9,938,375 (215^3) at s = 0.005 in a 2.5 x 1.2 x 1.2 m tank + 64 boxes

Kernel constants for all: h = 2 s, rho0 = 1000, gamma = 7, c0 = 20 m/s, alpha = 0.05,
eps = 0.5, g = -9.81, 10 substeps per 60 Hz tick, one Akinci layer on every wall box
(wall thickness 2 s). Positions are the reference lattice (origin + (i + 1/2) s, i outer,
k inner; crates/vxl-phys-fluid/src/fluid_access.rs:14-26) plus uniform jitter of +-1%
of the spacing from numpy's PCG64 with the scene seed; the particle mass is calibrated
on the unjittered lattice (fluid_access.rs:27-42).

All arithmetic that produces particle data is float32, in the reference's order, so
the oracle fed the same arrays sees the same inputs bit for bit.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import Params, make_params

F = np.float32

# Where the lattice-mass calibration and the Akinci body lattices come from. By default
# the library's own host code (vxl_sph_lattice_mass, vxl_sph_boundary_lattice); a
# caller that must not load the CUDA library (the CPU baseline) installs another source
# computing the same float32 values with use_lattice_source().
_LATTICE_SOURCE = None


def use_lattice_source(mass_fn=None, lattice_fn=None) -> None:
    """Install mass_fn(params, spacing) -> float and lattice_fn(shape, half, radius,
    spacing, h, layers) -> (points (N, 3) float32, volume); None restores the library's."""
    global _LATTICE_SOURCE
    _LATTICE_SOURCE = None if mass_fn is None else (mass_fn, lattice_fn)


def lattice_mass(params: Params, spacing: float) -> float:
    if _LATTICE_SOURCE is not None:
        return _LATTICE_SOURCE[0](params, spacing)
    from . import lattice_mass as lib_mass
    return lib_mass(params, spacing)


def boundary_lattice(shape: int, half, radius: float, spacing: float, h: float, layers: int):
    if _LATTICE_SOURCE is not None:
        return _LATTICE_SOURCE[1](shape, half, radius, spacing, h, layers)
    from . import boundary_lattice as lib_lattice
    return lib_lattice(shape, half, radius, spacing, h, layers)


@dataclass
class SceneSpec:
    name: str
    params: Params
    pos: np.ndarray      # (N_t, 3) float32, fluid prefix then boundary suffix
    vel: np.ndarray      # (N_t, 3) float32
    pmass: np.ndarray    # (N_t,) float32
    n_fluid: int
    spans: list          # [(body, origin(3), start, end)]
    spacing: float
    ticks: int
    meta: dict = field(default_factory=dict)

    @property
    def n_total(self) -> int:
        return int(self.pos.shape[0])

    @property
    def n_boundary(self) -> int:
        return self.n_total - self.n_fluid


def fluid_block(origin, dims, spacing) -> np.ndarray:
    """n0 x n1 x n2 lattice at origin + (i + 1/2) s, reference order (fluid_access.rs:16-26)."""
    s = F(spacing)
    i, j, k = np.meshgrid(np.arange(dims[0]), np.arange(dims[1]), np.arange(dims[2]), indexing="ij")
    out = np.empty((i.size, 3), F)
    for a, g in enumerate((i, j, k)):
        out[:, a] = F(origin[a]) + (g.reshape(-1).astype(F) + F(0.5)) * s
    return out


def jitter(pos: np.ndarray, spacing: float, seed: int, frac: float = 0.01) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    amp = F(frac) * F(spacing)
    return (pos + rng.uniform(-1.0, 1.0, size=pos.shape).astype(F) * amp).astype(F)


def _cross(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    # crates/vxl-phys-core/src/math.rs (Vec3::cross), float32 elementwise
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1).astype(F)


def rotate(q, v: np.ndarray) -> np.ndarray:
    """Quat::rotate_vec3: t = 2 (q x v); v + q x t + w t (float32)."""
    qv = np.broadcast_to(np.asarray(q[:3], F), v.shape)
    t = (_cross(qv, v) * F(2.0)).astype(F)
    return ((v + _cross(qv, t)) + t * F(q[3])).astype(F)


@dataclass
class Body:
    id: int
    half: tuple
    pos: tuple
    rot: tuple = (0.0, 0.0, 0.0, 1.0)
    linvel: tuple = (0.0, 0.0, 0.0)
    angvel: tuple = (0.0, 0.0, 0.0)


def body_particles(bodies, spacing: float, h: float, layers: int, rest_density: float, cache=None):
    """set_boundary_particles (crates/vxl-phys-fluid/src/fluid_step.rs:13-53) on the host:
    per-shape lattice (cached), world transform, surface velocity v + w x r, pmass = rho0 V_b,
    body-major layout; returns (pos, vel, pmass, spans relative to the boundary start)."""
    cache = {} if cache is None else cache
    ps, vs, ms, spans = [], [], [], []
    n = 0
    for b in bodies:
        key = tuple(np.asarray(b.half, F).tolist())
        if key not in cache:
            cache[key] = boundary_lattice(0, key, 0.0, spacing, h, layers)
        lat, vol = cache[key]
        if lat.shape[0] == 0:
            continue
        bp = np.asarray(b.pos, F)
        wp = (bp + rotate(b.rot, lat)).astype(F)
        r = (wp - bp).astype(F)
        wv = (np.asarray(b.linvel, F) + _cross(np.broadcast_to(np.asarray(b.angvel, F), r.shape), r)).astype(F)
        ps.append(wp)
        vs.append(wv)
        ms.append(np.full(wp.shape[0], F(rest_density) * F(vol), F))
        spans.append((b.id, tuple(float(x) for x in bp), n, n + wp.shape[0]))
        n += wp.shape[0]
    if not ps:
        return np.zeros((0, 3), F), np.zeros((0, 3), F), np.zeros(0, F), []
    return np.concatenate(ps), np.concatenate(vs), np.concatenate(ms), spans


def body_lattice(bodies, spacing: float, h: float, layers: int, cache=None):
    """The body-frame side of body_particles: (local points, body index into `bodies`) of
    the boundary segment in the same body-major order, for the device-side rebuild
    (vxl_sph_set_body_lattice + vxl_sph_set_body_poses)."""
    cache = {} if cache is None else cache
    pts, idx = [], []
    for q, b in enumerate(bodies):
        key = tuple(np.asarray(b.half, F).tolist())
        if key not in cache:
            cache[key] = boundary_lattice(0, key, 0.0, spacing, h, layers)
        lat, _ = cache[key]
        if lat.shape[0] == 0:
            continue
        pts.append(lat)
        idx.append(np.full(lat.shape[0], q, np.uint32))
    if not pts:
        return np.zeros((0, 3), F), np.zeros(0, np.uint32)
    return np.concatenate(pts).astype(F), np.concatenate(idx)


def floor_provider():
    """The fluid crate's FloorY test provider: solid half-space y < 0, bounds (-50, -1, -50)
    to (50, 0, 50) (crates/vxl-phys-fluid/src/tests.rs:9-44)."""
    from . import Faces
    return Faces([(1, 0.0, 1.0)], ((-50.0, -1.0, -50.0), (50.0, 0.0, 50.0)))


def tank_provider(half_width: float = 0.2):
    """The fluid crate's Tank test provider: floor y = 0 and four walls at x, z = +-0.2
    (half-spaces extending outward), bounds +-50 (crates/vxl-phys-fluid/src/tests.rs:46-110)."""
    from . import Faces
    w = half_width
    return Faces([(1, 0.0, 1.0), (0, -w, 1.0), (0, w, -1.0), (2, -w, 1.0), (2, w, -1.0)],
                 ((-50.0, -50.0, -50.0), (50.0, 50.0, 50.0)))


def box_obstacle(center, half):
    """A solid box as a convex half-space set (outward normals +-x, +-y, +-z)."""
    from . import Convex
    c, h = center, half
    planes = []
    for a in range(3):
        for sgn in (1.0, -1.0):
            n = [0.0, 0.0, 0.0]
            n[a] = sgn
            planes.append((tuple(n), float(F(F(sgn) * F(c[a])) + F(h[a]))))
    lo = tuple(float(F(c[a]) - F(h[a])) for a in range(3))
    hi = tuple(float(F(c[a]) + F(h[a])) for a in range(3))
    return Convex(planes, (lo, hi))


def box_mass_props(half, density: float):
    """Mass properties of a box body (crates/vxl-phys-core/src/mass.rs:35-48), float32 in the
    reference's order: m = rho ex ey ez with e = 2 half, I = m / 12 (e1^2 + e2^2); returns
    (inv_mass, local inverse inertia diagonal)."""
    rho = F(density) if density > 0 else F(1.0)
    ex, ey, ez = (F(2.0) * F(h) for h in half)
    m = F(F(F(rho * ex) * ey) * ez)
    ix = F(F(m / F(12.0)) * F(F(ey * ey) + F(ez * ez)))
    iy = F(F(m / F(12.0)) * F(F(ex * ex) + F(ez * ez)))
    iz = F(F(m / F(12.0)) * F(F(ex * ex) + F(ey * ey)))
    return F(F(1.0) / m), (F(F(1.0) / ix), F(F(1.0) / iy), F(F(1.0) / iz))


def tank_bodies(inner, t: float, first_id: int = 0) -> list:
    """Floor + four walls (static boxes) around the open box [0, inner]; thickness t
    (the reference's --tank pattern, gpu_tick_probe.rs:20-63, with the tank's own size)."""
    lx, ly, lz = (F(x) for x in inner)
    t = F(t)
    th = t * F(0.5)
    return [
        Body(first_id + 0, (lx * F(0.5) + t, th, lz * F(0.5) + t), (lx * F(0.5), -th, lz * F(0.5))),
        Body(first_id + 1, (th, ly * F(0.5), lz * F(0.5) + t), (-th, ly * F(0.5), lz * F(0.5))),
        Body(first_id + 2, (th, ly * F(0.5), lz * F(0.5) + t), (lx + th, ly * F(0.5), lz * F(0.5))),
        Body(first_id + 3, (lx * F(0.5) + t, ly * F(0.5), th), (lx * F(0.5), ly * F(0.5), -th)),
        Body(first_id + 4, (lx * F(0.5) + t, ly * F(0.5), th), (lx * F(0.5), ly * F(0.5), lz + th)),
    ]


def closed_tank_bodies(inner, t: float, first_id: int = 0) -> list:
    """tank_bodies plus a lid over [0, inner] (a sixth static box at y = ly): the batched
    and served tanks run for hundreds of ticks with the reference constants, whose
    acoustic CFL number c0 dt / h exceeds 1 at most spacings, and the lid keeps
    splashing particles inside the tank."""
    lx, ly, lz = (F(x) for x in inner)
    t = F(t)
    th = t * F(0.5)
    lid = Body(first_id + 5, (lx * F(0.5) + t, th, lz * F(0.5) + t), (lx * F(0.5), ly + th, lz * F(0.5)))
    return tank_bodies(inner, t, first_id) + [lid]


def baseline_params(spacing: float, substeps: int = 10, layers: int = 1, **over) -> Params:
    kw = dict(rest_density=1000.0, smoothing_radius=2.0 * spacing, xsph_viscosity=0.5, sound_speed=20.0,
              gamma_tait=7.0, substeps=substeps, boundary_layers=layers, gravity=(0.0, -9.81, 0.0),
              max_speed_frac=0.4, artificial_viscosity=0.05)
    kw.update(over)
    p = make_params(**kw)
    p.particle_mass = lattice_mass(p, spacing)
    return p


def assemble(name, params, fluid_pos, bodies, spacing, ticks, meta=None, cache=None) -> SceneSpec:
    nf = fluid_pos.shape[0]
    bpos, bvel, bm, bspans = body_particles(bodies, spacing, params.smoothing_radius, params.boundary_layers,
                                            params.rest_density, cache)
    pos = np.concatenate([fluid_pos, bpos]).astype(F)
    vel = np.zeros_like(pos)
    vel[nf:] = bvel
    pm = np.concatenate([np.full(nf, F(params.particle_mass), F), bm]).astype(F)
    spans = [(b, o, s + nf, e + nf) for (b, o, s, e) in bspans]
    return SceneSpec(name, params, pos, vel, pm, nf, spans, spacing, ticks, meta or {})


def dam_break(name: str, dims, spacing: float, tank, ticks: int, seed: int, extra_bodies=(), substeps: int = 10,
              layers: int = 1, **over) -> SceneSpec:
    params = baseline_params(spacing, substeps=substeps, layers=layers, **over)
    fluid = jitter(fluid_block((0.0, 0.0, 0.0), dims, spacing), spacing, seed)
    walls = tank_bodies(tank, 2.0 * spacing)
    bodies = walls + list(extra_bodies)
    fill = float(np.prod(np.asarray(dims) * spacing) / np.prod(tank))
    return assemble(name, params, fluid, bodies, spacing, ticks,
                    {"dims": tuple(dims), "tank": tuple(tank), "fill": fill, "seed": seed, "bodies": bodies,
                     "dynamic": [False] * len(walls) + [True] * len(extra_bodies)})


def floating_boxes(n: int, seed: int, lo, hi, half_lo: float, half_hi: float, first_id: int, gap: float) -> list:
    """n boxes with per-axis half extents U(half_lo, half_hi) at non-overlapping random
    centres inside [lo, hi] (seeded rejection sampling)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out, boxes = [], []
    tries = 0
    while len(out) < n and tries < 100000:
        tries += 1
        half = rng.uniform(half_lo, half_hi, 3).astype(F)
        c = np.array([rng.uniform(lo[a] + half[a], hi[a] - half[a]) for a in range(3)], F)
        if any(np.all(np.abs(c - c2) < half + h2 + gap) for c2, h2 in boxes):
            continue
        boxes.append((c, half))
        out.append(Body(first_id + len(out), tuple(float(x) for x in half), tuple(float(x) for x in c)))
    return out


def dam0(seed: int = 0) -> SceneSpec:
    return dam_break("dam0", (16, 32, 32), 0.02, (1.0, 0.64, 0.64), 600, seed)


def dam1(seed: int = 1) -> SceneSpec:
    return dam_break("dam1", (100, 100, 100), 0.01, (2.0, 2.0, 1.0), 300, seed)


def dam10m(seed: int = 2, boxes: int = 64) -> SceneSpec:
    extra = floating_boxes(boxes, seed + 1000, (1.2, 0.05, 0.05), (2.45, 1.1, 1.15), 0.025, 0.075, 5, 0.02)
    return dam_break("dam10m", (215, 215, 215), 0.005, (2.5, 1.2, 1.2), 120, seed, extra_bodies=extra)


def dam10m_block(n: int = 100, seed: int = 2, boxes: int = 64) -> SceneSpec:
    """The dam10m tank, walls and boxes with an n^3 fluid block instead of 215^3: the grid
    box is still the tank's, so the bins are still doubled to 2h (64 particles per cell in the
    block), at a size a profiler can capture."""
    extra = floating_boxes(boxes, seed + 1000, (1.2, 0.05, 0.05), (2.45, 1.1, 1.15), 0.025, 0.075, 5, 0.02)
    return dam_break(f"dam10m_block{n}", (n, n, n), 0.005, (2.5, 1.2, 1.2), 120, seed, extra_bodies=extra)


def dam10m_sample(n: int = 100, seed: int = 2) -> SceneSpec:
    """A bounded sample of dam10m for the CPU baseline: an n^3 fluid block in the corner of
    the dam10m tank with the tank's floor and two corner walls cropped to the block's
    surroundings, so the boundary-to-fluid ratio is close to the full scene's (0.11), and two
    small marker boxes at the tank's far corners, so the grid box, and with it the doubled
    bins, is the full scene's. Same spacing, constants and jitter rule; the boxes of the full
    scene lie far from the block and are left out."""
    s = 0.005
    t = F(2.0 * s)
    th = t * F(0.5)
    ext = F((n + 8) * s)  # the block plus a margin of 8 spacings
    bodies = [
        Body(0, (ext * F(0.5) + t, th, ext * F(0.5) + t), (ext * F(0.5), -th, ext * F(0.5))),  # floor
        Body(1, (th, ext * F(0.5), ext * F(0.5) + t), (-th, ext * F(0.5), ext * F(0.5))),      # x = 0 wall
        Body(3, (ext * F(0.5) + t, ext * F(0.5), th), (ext * F(0.5), ext * F(0.5), -th)),      # z = 0 wall
        Body(5, (s, s, s), (2.5 + th, 1.2 - s, 1.2 + th)),                                      # far corner markers
        Body(6, (s, s, s), (2.5 + th, -th, -th)),
    ]
    params = baseline_params(s)
    fluid = jitter(fluid_block((0.0, 0.0, 0.0), (n, n, n), s), s, seed)
    fill = float((n * s) ** 3 / (2.5 * 1.2 * 1.2))
    return assemble(f"dam10m_sample{n}", params, fluid, bodies, s, 120,
                    {"dims": (n, n, n), "tank": (2.5, 1.2, 1.2), "fill": fill, "seed": seed, "bodies": bodies,
                     "dynamic": [False] * len(bodies)})


def small_dam(n=(8, 8, 8), spacing: float = 0.05, tank=(0.8, 0.6, 0.6), seed: int = 3, substeps: int = 4,
              ticks: int = 10, **over) -> SceneSpec:
    """A small tank scene for parity tests (same construction, smaller sizes)."""
    return dam_break("small", n, spacing, tank, ticks, seed, substeps=substeps, **over)


def tank_scene(kind: str, n_target: int, spacing: float, aspect: float, fill: float, seed: int,
               ticks: int = 300, substeps: int = 10, closed: bool = True, name: str | None = None) -> SceneSpec:
    """One tank of the batched and served workloads. The tank (W, H, D) = (aspect L, L, L)
    holds n_target s^3 / fill of volume; the fluid (about n_target particles) is either a
    dam-break column over the full depth at the x = 0 end, 0.9 H tall, or a sloshing layer
    over the whole floor (fill H deep) with horizontal velocity u = U0 sin(pi x / W),
    U0 ~ U(0.2, 0.6) m/s from the seed. Spacing s is rounded to float32; h = 2 s."""
    s = float(F(spacing))
    vol = n_target * s ** 3 / fill
    L = (vol / aspect) ** (1.0 / 3.0)
    W, H, D = aspect * L, L, L
    nz = max(1, int(D / s))
    if kind == "dam":
        ny = max(1, int(0.9 * H / s))
        nx = max(1, int(round(n_target / (ny * nz))))
        nx = min(nx, max(1, int(W / s)))
    elif kind == "slosh":
        nx = max(1, int(W / s))
        ny = max(1, min(int(round(n_target / (nx * nz))), int(0.9 * H / s)))
    else:
        raise ValueError(kind)
    tank = (float(F(W)), float(F(H)), float(F(D)))
    params = baseline_params(s, substeps=substeps)
    fluid = jitter(fluid_block((0.0, 0.0, 0.0), (nx, ny, nz), s), s, seed)
    walls = (closed_tank_bodies if closed else tank_bodies)(tank, 2.0 * s)
    meta = {"kind": kind, "dims": (nx, ny, nz), "tank": tank, "fill": float(nx * ny * nz * s ** 3 / (W * H * D)),
            "aspect": aspect, "seed": seed, "closed": closed}
    spec = assemble(name or f"{kind}{n_target}", params, fluid, walls, s, ticks, meta)
    if kind == "slosh":
        rng = np.random.Generator(np.random.PCG64(seed + 7919))
        u0 = F(rng.uniform(0.2, 0.6))
        x = spec.pos[:spec.n_fluid, 0]
        spec.vel[:spec.n_fluid, 0] = (u0 * np.sin(F(np.pi) * x / F(W)).astype(F)).astype(F)
        spec.meta["u0"] = float(u0)
    return spec


def _log_uniform_int(rng, lo: int, hi: int) -> int:
    return int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))


def batched_mix(n_scenes: int = 256, seed: int = 7, n_lo: int = 4096, n_hi: int = 262144,
                ticks: int = 300, substeps: int = 10) -> list:
    """The batched workload: n_scenes independent dam-break tanks with particle counts
    log-uniform in [n_lo, n_hi], aspect U(0.5, 2), fill U(0.2, 0.6) and spacing
    U(0.005, 0.02) m (h = 2 s), all drawn from one seed (PCG64); each scene's jitter seed
    is seed * 100003 + its index."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for q in range(n_scenes):
        n = _log_uniform_int(rng, n_lo, n_hi)
        aspect = float(rng.uniform(0.5, 2.0))
        fill = float(rng.uniform(0.2, 0.6))
        s = float(rng.uniform(0.005, 0.02))
        out.append(tank_scene("dam", n, s, aspect, fill, seed * 100003 + q, ticks, substeps, name=f"mix{q}"))
    return out


@dataclass
class Request:
    arrival_s: float
    spec: SceneSpec
    ticks: int


def served_stream(n_requests: int, rate: float, seed: int = 11, n_lo: int = 8192, n_hi: int = 1048576,
                  ticks_lo: int = 60, ticks_hi: int = 600, tick_scale: float = 1.0, substeps: int = 10) -> list:
    """The served workload: requests arriving as a Poisson process of `rate` per second,
    particle counts log-uniform in [n_lo, n_hi], ticks uniform in [ticks_lo, ticks_hi]
    (times tick_scale, at least 1), a dam-break or sloshing tank (even odds) with aspect,
    fill and spacing drawn as in batched_mix, each from its own per-request seed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for r in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        n = _log_uniform_int(rng, n_lo, n_hi)
        ticks = max(1, int(round(int(rng.integers(ticks_lo, ticks_hi + 1)) * tick_scale)))
        kind = "dam" if rng.uniform() < 0.5 else "slosh"
        aspect = float(rng.uniform(0.5, 2.0))
        fill = float(rng.uniform(0.2, 0.6))
        s = float(rng.uniform(0.005, 0.02))
        spec = tank_scene(kind, n, s, aspect, fill, seed * 1000003 + r, ticks, substeps, name=f"req{r}")
        out.append(Request(t, spec, ticks))
    return out


CONFIGS = {"dam0": dam0, "dam1": dam1, "dam10m": dam10m}
