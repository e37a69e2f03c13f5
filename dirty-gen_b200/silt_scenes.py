"""Seeded synthetic scenes for the sheet step (no dataset exists for this path).

Each builder returns float32 host arrays, row-major j*res + i, that the caller
feeds to the sheet API (map_water_bed, lay_slurry_mask, read_substrate_grid):

* window200 -- a 200 x 200 window of 0.2 m cells: 4-octave value-noise bed,
  0.3 m amplitude, a rut pair (0.15 m deep, 0.25 m wide, 1.5 m apart), a
  Gaussian puddle (0.10 m peak, cut at 3 m) and a clay slurry film of one
  seeded depth in 0.02..0.05 m inside the ruts.
* grid -- the same bed noise on a large grid with eight seeded puddles
  (0.05..0.2 m deep, radius 2..8 m), plus four tires in a 1.5 m x 2.4 m
  rectangle driving +z and an inflow strip on row 0.
* batch_windows -- many independent windows of log-uniform sides (64..512
  cells), each a `grid` scene with its own seed, 1..4 puddles and 0..4 tires.

The value noise is the reference's `hash01`/`relief_value`
(src/fluid_core.rs:4639-4668) evaluated in float32.
"""
import numpy as np

F = np.float32
CLAY, SILT, SAND, WATER, OTHER = 0, 1, 2, 3, 4


def hash01(ix, iz, seed):
    """src/fluid_core.rs:4639-4648 with u32 wrapping arithmetic."""
    ix = np.asarray(ix).astype(np.int64).astype(np.uint32)
    iz = np.asarray(iz).astype(np.int64).astype(np.uint32)
    with np.errstate(over="ignore"):
        n = (ix * np.uint32(0x27BB2EE6) + iz * np.uint32(0x165667B1)) ^ np.uint32(seed & 0xFFFFFFFF)
        n = n * np.uint32(0x9E3779B1)
        n ^= n >> np.uint32(16)
        n = n * np.uint32(0x85EBCA6B)
        n ^= n >> np.uint32(13)
    return (n >> np.uint32(8)).astype(F) * F(1.0 / 16777216.0)


def relief_value(x, z, seed):
    """src/fluid_core.rs:4651-4668, value noise in -1..1."""
    x = np.asarray(x, F)
    z = np.asarray(z, F)
    x0 = np.floor(x)
    z0 = np.floor(z)
    fx = x - x0
    fz = z - z0
    sx = fx * fx * (F(3.0) - F(2.0) * fx)
    sz = fz * fz * (F(3.0) - F(2.0) * fz)
    ix = x0.astype(np.int64)
    iz = z0.astype(np.int64)
    v00 = hash01(ix, iz, seed)
    v10 = hash01(ix + 1, iz, seed)
    v01 = hash01(ix, iz + 1, seed)
    v11 = hash01(ix + 1, iz + 1, seed)
    a = v00 + (v10 - v00) * sx
    b = v01 + (v11 - v01) * sx
    return (a + (b - a) * sz) * F(2.0) - F(1.0)


def bed_noise(x, z, seed):
    """0.3 m x sum over 4 octaves of 0.5^o relief_value(x 0.25 2^o, z 0.25 2^o, seed+o) / 1.875."""
    acc = np.zeros(np.broadcast(x, z).shape, F)
    for o in range(4):
        f = F(0.25 * 2.0 ** o)
        acc += F(0.5 ** o) * relief_value(x * f, z * f, (seed + o) & 0xFFFFFFFF)
    return F(0.3) * acc / F(1.875)


def snap_origin(cx, cz, extent, cell):
    """src/fluid_core.rs:9888-9892."""
    x = F(cx) - F(extent) * F(0.5)
    z = F(cz) - F(extent) * F(0.5)
    return np.floor(x / F(cell)) * F(cell), np.floor(z / F(cell)) * F(cell)


def cell_centres(res, cell, origin):
    i = np.arange(res, dtype=F)
    x = origin[0] + (i + F(0.5)) * F(cell)
    z = origin[1] + (i + F(0.5)) * F(cell)
    return np.meshgrid(x, z)  # [j, i]


def _rng(seed):
    return np.random.default_rng(seed & 0xFFFFFFFF)


def rut_profile(x, centres=(-0.75, 0.75), depth=0.15, half_width=0.125):
    """Cosine rut cross-section; returns (lowering of the bed, inside-rut mask)."""
    low = np.zeros_like(x, dtype=F)
    inside = np.zeros(x.shape, bool)
    for c in centres:
        d = np.abs(x - F(c))
        m = d < F(half_width)
        low = np.where(m, np.maximum(low, F(depth) * F(0.5) * (F(1.0) + np.cos(F(np.pi) * d / F(half_width)))), low)
        inside |= m
    return low.astype(F), inside


def window200(seed=0x9E3779B9, res=200, cell=0.2, center=(0.0, 0.0)):
    extent = res * cell
    origin = snap_origin(center[0], center[1], extent, cell)
    x, z = cell_centres(res, cell, origin)
    bed = bed_noise(x, z, seed)
    low, ruts = rut_profile(x)
    bed = bed - low
    r2 = (x - F(center[0])) ** 2 + (z - F(center[1])) ** 2
    water = np.where(r2 < F(9.0), F(0.10) * np.exp(-r2 / F(2.0)), F(0.0)).astype(F)
    s = _rng(seed).uniform(0.02, 0.05)
    slurry = np.where(ruts, F(s), F(0.0)).astype(F)
    return dict(res=res, cell=cell, origin=origin, center=center, bed=bed.ravel(), water=water.ravel(),
                slurry=slurry.ravel(), slurry_grain=CLAY, slurry_moisture=0.55,
                moisture=np.full(res * res, 0.55, F), grain=np.full(res * res, CLAY, np.uint8))


def grid(res=2048, cell=0.2, seed=0x9E3779B9, puddles=8, center=(0.0, 0.0)):
    extent = res * cell
    origin = snap_origin(center[0], center[1], extent, cell)
    x, z = cell_centres(res, cell, origin)
    bed = bed_noise(x, z, seed)
    rng = _rng(seed + 1)
    water = np.zeros_like(bed)
    half = F(extent * 0.5)
    for _ in range(puddles):
        d = F(rng.uniform(0.05, 0.2))
        rad = F(rng.uniform(2.0, 8.0))
        px = F(center[0]) + F(rng.uniform(-1.0, 1.0)) * (half - rad)
        pz = F(center[1]) + F(rng.uniform(-1.0, 1.0)) * (half - rad)
        r2 = (x - px) ** 2 + (z - pz) ** 2
        bowl = np.where(r2 < rad * rad, d * (F(1.0) - r2 / (rad * rad)), F(0.0)).astype(F)
        water = np.maximum(water, bowl)
    low, ruts = rut_profile(x - F(center[0]))
    bed = bed - low
    slurry = np.where(ruts & (np.abs(z - F(center[1])) < F(20.0)), F(rng.uniform(0.02, 0.05)), F(0.0)).astype(F)
    return dict(res=res, cell=cell, origin=origin, center=center, bed=bed.ravel(), water=water.ravel(),
                slurry=slurry.ravel(), slurry_grain=CLAY, slurry_moisture=0.55,
                moisture=np.full(res * res, 0.55, F), grain=np.full(res * res, CLAY, np.uint8))


def basin(res=200, cell=0.2, level=0.3, speed=0.75, seed=0x9E3779B9, center=(0.0, 0.0)):
    """Open water: a flat sand floor in a 12 m square with 0.6 banks, a little
    bed noise, water to `level`, and a current of `speed` m/s along +x in the
    band |z| < 3 m (the basin of the reference's open-water tests)."""
    extent = res * cell
    origin = snap_origin(center[0], center[1], extent, cell)
    x, z = cell_centres(res, cell, origin)
    d = np.maximum(np.maximum(np.abs(x) - F(6.0), np.abs(z) - F(6.0)), F(0.0))
    bed = (d * F(0.6) + F(0.1) * bed_noise(x, z, seed)).astype(F)
    water = np.maximum(F(level) - bed, F(0.0)).astype(F)
    u = np.where((np.abs(z) < F(3.0)) & (water > F(0.0)), F(speed), F(0.0)).astype(F)
    v = np.zeros_like(u)
    n = res * res
    return dict(res=res, cell=cell, origin=origin, center=center, bed=bed.ravel(), water=water.ravel(),
                u=u.ravel(), v=v.ravel(), moisture=np.full(n, 0.9, F), grain=np.full(n, SAND, np.uint8))


def channel(res=200, cell=0.2, level=0.3, speed=0.5, seed=0x9E3779B9, center=(0.0, 0.0)):
    """A river channel along x through the whole window: flat sand floor for
    |z| < 4 m, banks rising 0.6 per metre beyond, a little bed noise, water
    to `level` and a current of `speed` m/s along +x."""
    extent = res * cell
    origin = snap_origin(center[0], center[1], extent, cell)
    x, z = cell_centres(res, cell, origin)
    bed = (np.maximum(np.abs(z) - F(4.0), F(0.0)) * F(0.6) + F(0.05) * bed_noise(x, z, seed)).astype(F)
    water = np.maximum(F(level) - bed, F(0.0)).astype(F)
    u = np.where(water > F(0.0), F(speed), F(0.0)).astype(F)
    n = res * res
    return dict(res=res, cell=cell, origin=origin, center=center, bed=bed.ravel(), water=water.ravel(),
                u=u.ravel(), v=np.zeros(n, F), moisture=np.full(n, 0.9, F), grain=np.full(n, SAND, np.uint8))


def seed_basin(core, scene):
    """Seeds a sheet handle (oracle or device) with a basin scene."""
    core.read_substrate(scene["bed"], scene["moisture"], scene["grain"])
    core.map_grain(scene["grain"])
    core.map_water_bed(scene["bed"], scene["water"])
    core.map_water_velocity(scene["u"], scene["v"])


def tires_at(t, speed=5.0, center=(0.0, 0.0), track=1.5, wheelbase=2.4, radius=0.38, width=0.2, slip=0.3,
             z0=-10.0):
    """Four tires in a track x wheelbase rectangle driving +z at `speed`."""
    zc = F(center[1]) + F(z0) + F(speed) * F(t)
    out = []
    for dx, dz in ((-0.5, -0.5), (0.5, -0.5), (-0.5, 0.5), (0.5, 0.5)):
        out.append(dict(x=float(F(center[0]) + F(dx * track)), z=float(zc + F(dz * wheelbase)), forward_x=0.0,
                        forward_z=1.0, radius=radius, width=width, speed=speed, slip=slip))
    return out


def vehicle_bodies(x=0.1, z=0.4, yaw=0.35):
    """A vehicle standing in the window as HydroSolid bodies (the shapes of
    the reference's Vehicle::hydro_solids, src/vehicle.rs:345-386): the belly
    (a 2.3 x 1.4 m wall) and four wheel contacts (0.5 x 0.3 m footprints,
    radius 0.38, width 0.2), undersides below the bed."""
    belly = dict(x=x, z=z, yaw=yaw, half_length=1.15, half_width=0.70, bottom_y=-1.0, top_y=2.0, contact=0)
    wheels = [dict(x=x + dx, z=z + dz, yaw=yaw, half_length=0.25, half_width=0.15, bottom_y=-1.0, top_y=2.0,
                   contact=1, radius=0.38, width=0.2) for dx in (-0.75, 0.75) for dz in (-1.2, 1.2)]
    return [belly] + wheels


def seed_walled(core, scene, u=0.15, v=0.45):
    """The walled config-1 window: the scene, a uniform current and the
    vehicle's bodies."""
    seed_core(core, scene)
    n = scene["res"] * scene["res"]
    core.map_water_velocity(np.full(n, u, np.float32), np.full(n, v, np.float32))
    core.set_hydro_solids(vehicle_bodies())


def seed_core(core, scene):
    """Seeds a sheet handle (oracle or device) the same way: bed + water, the
    rut slurry, then the substrate read that fixes moisture and grain."""
    core.map_water_bed(scene["bed"], scene["water"])
    core.lay_slurry_mask(scene["slurry"], scene["slurry_grain"], scene["slurry_moisture"])
    core.read_substrate(scene["bed"], scene["moisture"], scene["grain"])


def batch_windows(n=256, base_seed=0x9E3779B9, cell=0.2, lo=64, hi=512):
    """Window k: side round(exp(U(ln lo, ln hi))), seed base_seed + k, 1..4
    puddles and 0..4 tires (the first of tires_at's four)."""
    rng = _rng(base_seed + 7)
    out = []
    for k in range(n):
        side = int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi))))))
        puddles = int(rng.integers(1, 5))
        tires = int(rng.integers(0, 5))
        sc = grid(res=side, cell=cell, seed=base_seed + k, puddles=puddles)
        sc["tires"] = tires
        out.append(sc)
    return out
