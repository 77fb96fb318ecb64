"""Seeded synthetic MPM scenes and the per-substep parameter record.

Every scene is generated from a counter-based SplitMix64 stream, so the oracle
and the CUDA engine see bit-identical inputs.  Records mirror the reference's
host structs:

* ``MATERIAL_DTYPE`` -- ``MaterialParams`` (src/core/MaterialParams.h:16-38)
* ``COLLIDER_DTYPE`` -- ``ColliderPrimitive`` (src/core/Collider.h:19-29)
* ``FORCE_DTYPE``    -- ``ForceGPU`` (src/core/Force.h:27-32)

``StepParams`` carries the scalar fields of ``MPMSimPC`` (src/core/MPMSimPC.h:14-77)
that the substep reads, built like ``MPMEngine::buildPC`` (src/engine/MPMEngine.cpp:356-400).

The workloads are synthetic stand-ins with the shapes and value ranges of the
five measured configurations: an elastic block, a jelly/sand multimaterial
scene, a 1M-particle Drucker-Prager slope over a terrain SDF, a 64-scene mix,
and a differentiable elastic block.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MAT_ELASTIC, MAT_VON_MISES, MAT_DRUCKER_PRAGER, MAT_GRANULAR_POWDER, MAT_FLUID, MAT_VISCOPLASTIC_MUD, MAT_FIXED_COROTATED = range(7)
COLL_PLANE, COLL_SPHERE, COLL_BOX, COLL_CAPSULE = range(4)
FORCE_GRAVITY, FORCE_CONSTANT_WIND = 0, 1

MATERIAL_DTYPE = np.dtype([
    ("mu", "<f4"), ("lambda", "<f4"), ("rho0", "<f4"), ("model", "<u4"),
    ("M_friction", "<f4"), ("q_cohesion", "<f4"), ("q_max", "<f4"), ("bulkK", "<f4"),
    ("fluidGamma", "<f4"), ("viscosity", "<f4"), ("hardening", "<f4"), ("xi", "<f4"),
    ("pad", "<f4", (4,)),
])
COLLIDER_DTYPE = np.dtype([
    ("type", "<u4"), ("pos", "<f4", (3,)), ("nrm", "<f4", (3,)), ("radius", "<f4"),
    ("vel", "<f4", (3,)), ("restitution", "<f4"), ("friction", "<f4"), ("pad", "<f4", (3,)),
])
FORCE_DTYPE = np.dtype([("type", "<u2"), ("affectMask", "<u2"), ("data", "<f4", (7,))])
# nebula_mpm_emitter: the MPM fields of Emitter (src/core/Emitter.h:39-82)
EMITTER_DTYPE = np.dtype([
    ("shape", "<u4"), ("center", "<f4", (3,)), ("size", "<f4", (3,)), ("vel", "<f4", (3,)), ("center_vel", "<f4", (3,)),
    ("particles_per_step", "<i4"), ("particleType", "<u4"), ("emitAlongNormal", "<u4"), ("velocityRandomness", "<f4"),
    ("step_count", "<i4"), ("particleVolume", "<f4"), ("pad", "<u4"),
])
EMIT_AABB, EMIT_SPHERE, EMIT_ELLIPSE = range(3)
assert MATERIAL_DTYPE.itemsize == 64 and COLLIDER_DTYPE.itemsize == 64 and FORCE_DTYPE.itemsize == 32

FIELDS = ("P", "v", "F0", "F1", "F2", "B0", "B1", "B2")


# ----------------------------------------------------------------------------- RNG
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """n counter-based SplitMix64 outputs for (seed, stream): value i mixes
    seed*2^32 + stream*2^48... (plus (i+1) golden-ratio increments)."""
    with np.errstate(over="ignore"):
        base = np.uint64((seed * 0x100000001B3 + stream * 0xD1B54A32D192ED03) & 0xFFFFFFFFFFFFFFFF)
        z = base + (np.arange(1, n + 1, dtype=np.uint64) * _GOLDEN)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int, stream: int = 0, lo=0.0, hi=1.0) -> np.ndarray:
    """float64 uniforms in [lo, hi) from the top 53 bits of SplitMix64."""
    u = (splitmix64(seed, n, stream) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


# ----------------------------------------------------------------------------- domain
def grid_res(domain_size, cell_size):
    """domain::gridRes (src/core/Domain.h:14-17): max(1, ceil(size / h)) in float32."""
    ds = np.asarray(domain_size, np.float32)
    h = np.float32(max(np.float32(cell_size), np.float32(1e-6)))
    r = np.ceil(ds / h)
    return tuple(int(max(1, v)) for v in r)


def morton_cube_res(res):
    """domain::mortonCubeRes (src/core/Domain.h:25-30): next pow2 >= max axis."""
    m = max(max(res), 1)
    p = 1
    while p < m:
        p <<= 1
    return p


def hash_cells(res):
    """domain::hashCells (src/core/Domain.h:34-37): cubeRes^3."""
    c = morton_cube_res(res)
    return c * c * c


def n_groups(cells):
    return (cells + 255) // 256


def _expand(v):
    v = v.astype(np.uint64)
    v = (v | (v << np.uint64(16))) & np.uint64(0x030000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x0300F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x030C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x09249249)
    return v


def morton_encode(x, y, z):
    """Vectorised Morton code x | y<<1 | z<<2 (mpm_common.glsl:178-181)."""
    x = np.asarray(x)
    return (_expand(x) | (_expand(np.asarray(y)) << np.uint64(1)) | (_expand(np.asarray(z)) << np.uint64(2))).astype(np.uint32)


def lame(E, nu):
    """calcMu / calcLambda (src/core/MaterialParams.h:42-43), float32."""
    E = np.float32(E)
    nu = np.float32(nu)
    mu = E / (np.float32(2.0) * (np.float32(1.0) + nu))
    lam = E * nu / ((np.float32(1.0) + nu) * (np.float32(1.0) - np.float32(2.0) * nu))
    return float(mu), float(lam)


def material(model, E, nu, rho0, M_friction=0.0, q_cohesion=0.0, q_max=1e5, bulkK=0.0, viscosity=0.0):
    m = np.zeros(1, MATERIAL_DTYPE)
    mu, lam = lame(E, nu)
    m["mu"], m["lambda"], m["rho0"], m["model"] = mu, lam, rho0, model
    m["M_friction"], m["q_cohesion"], m["q_max"], m["bulkK"], m["viscosity"] = M_friction, q_cohesion, q_max, bulkK, viscosity
    return m[0]


# The reference's presets (src/core/MaterialParams.h:46-103), same parameters.
def preset_jelly(E=1e4, nu=0.4, rho0=1000.0):
    return material(MAT_ELASTIC, E, nu, rho0)


def preset_sand(E=1e5, nu=0.3, rho0=1600.0):
    return material(MAT_DRUCKER_PRAGER, E, nu, rho0, M_friction=0.577)


def preset_water(rho0=1000.0, bulkK=5e3):
    m = material(MAT_FLUID, 0.0, 0.0, rho0, bulkK=bulkK, viscosity=0.01)
    m["mu"], m["lambda"], m["fluidGamma"] = 0.0, 0.0, 7.0
    return m


def preset_mud(E=8e4, nu=0.35, rho0=1800.0):
    return material(MAT_VISCOPLASTIC_MUD, E, nu, rho0, M_friction=0.4, q_cohesion=5e2, viscosity=0.1)


def preset_powder(E=5e4, nu=0.25, rho0=1200.0):
    return material(MAT_GRANULAR_POWDER, E, nu, rho0, M_friction=0.8, q_cohesion=50.0)


def emitter(shape, center, size, vel=(0, 0, 0), particles_per_step=1024, particle_type=1, step_count=-1, center_vel=(0, 0, 0),
            along_normal=False, randomness=0.0, particle_volume=0.0):
    """An emitter record (defaults as Emitter, src/core/Emitter.h:41-62)."""
    e = np.zeros(1, EMITTER_DTYPE)
    e["shape"], e["center"][0], e["size"][0], e["vel"][0] = shape, center, size, vel
    e["center_vel"][0], e["particles_per_step"], e["particleType"] = center_vel, particles_per_step, particle_type
    e["emitAlongNormal"], e["velocityRandomness"], e["step_count"], e["particleVolume"] = int(along_normal), randomness, step_count, particle_volume
    return e[0]


def aabb_emitter(lo, hi, vel, particles_per_step, **kw):
    """AABBEmitter::FromAABB (Emitter.h:136-143)."""
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    return emitter(EMIT_AABB, (lo + hi) * np.float32(0.5), hi - lo, vel, particles_per_step, **kw)


def sphere_emitter(center, radius, vel, particles_per_step, **kw):
    """SphereEmitter::FromSphere (Emitter.h:184-191)."""
    return emitter(EMIT_SPHERE, center, (radius, radius, radius), vel, particles_per_step, **kw)


def ellipse_emitter(center, semi_a, semi_b, vel, particles_per_step, **kw):
    """EllipseEmitter's sample() convention: semi-axes along x and y, z fixed."""
    return emitter(EMIT_ELLIPSE, center, (semi_a, semi_b, 0.0), vel, particles_per_step, **kw)


def gravity(g=(0.0, -9.8, 0.0)):
    """A GravityForce record with direction (0,1,0)-style packing: dir=g/|g|, strength=|g|."""
    f = np.zeros(1, FORCE_DTYPE)
    g = np.asarray(g, np.float64)
    s = float(np.linalg.norm(g))
    f["type"] = FORCE_GRAVITY
    f["data"][0, :3] = g / s if s > 0 else 0.0
    f["data"][0, 3] = s
    return f[0]


def wind(direction=(1.0, 0.0, 0.0), strength=1.0, affect_mask=0):
    """A ConstantWindForce record (Force.h:152-170): v += dir * strength * dt on
    grid nodes; affect_mask 0 = every engine, else bit 0 selects MPM."""
    f = np.zeros(1, FORCE_DTYPE)
    f["type"] = FORCE_CONSTANT_WIND
    f["affectMask"] = affect_mask
    f["data"][0, :3] = direction
    f["data"][0, 3] = strength
    return f[0]


def sphere_collider(center, radius, vel=(0, 0, 0), restitution=0.3, friction=0.0):
    c = np.zeros(1, COLLIDER_DTYPE)
    c["type"] = COLL_SPHERE
    c["pos"][0] = center
    c["radius"] = radius
    c["vel"][0] = vel
    c["restitution"], c["friction"] = restitution, friction
    return c[0]


@dataclass
class StepParams:
    """Scalar parameters of one substep (the MPMSimPC fields the kernels read)."""
    dt: float
    cell_size: float
    domain_size: tuple
    world_min: tuple = (0.0, 0.0, 0.0)
    flip_ratio: float = -1.0
    materials: list = field(default_factory=list)
    colliders: list = field(default_factory=list)
    forces: list = field(default_factory=list)
    mu_lame: float = 0.0
    lambda_lame: float = 0.0
    rho0: float = 1000.0
    M_friction: float = 0.577
    q_cohesion: float = 0.0
    q_max: float = 1e5
    plastic_model: int = 0

    @property
    def grid_res(self):
        return grid_res(self.domain_size, self.cell_size)

    @property
    def cube_res(self):
        return morton_cube_res(self.grid_res)

    @property
    def hash_cells(self):
        return hash_cells(self.grid_res)

    @property
    def world_max(self):
        return tuple(float(np.float32(a) + np.float32(b)) for a, b in zip(self.world_min, self.domain_size))

    def materials_array(self):
        a = np.zeros(max(1, len(self.materials)), MATERIAL_DTYPE)
        for i, m in enumerate(self.materials):
            a[i] = m
        return a

    def colliders_array(self):
        a = np.zeros(max(1, len(self.colliders)), COLLIDER_DTYPE)
        for i, c in enumerate(self.colliders):
            a[i] = c
        return a

    def forces_array(self):
        a = np.zeros(max(1, len(self.forces)), FORCE_DTYPE)
        for i, f in enumerate(self.forces):
            a[i] = f
        return a


@dataclass
class Scene:
    name: str
    params: StepParams
    state: dict
    substeps: int
    sdf: np.ndarray | None = None
    extra: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.state["P"].shape[0]


def make_state(pos, vp, vel=None, mat_ids=None) -> dict:
    """Particle state in the reference layout (MPMEngine.cpp:46-53): 8 float4 per
    particle; v.w carries the material id bits, F = I, B = 0, stress = 0."""
    n = pos.shape[0]
    st = {f: np.zeros((n, 4), np.float32) for f in FIELDS}
    st["P"][:, :3] = pos
    st["P"][:, 3] = vp
    if vel is not None:
        st["v"][:, :3] = vel
    ids = np.zeros(n, np.uint32) if mat_ids is None else np.asarray(mat_ids, np.uint32)
    st["v"][:, 3] = ids.view(np.float32)
    st["F0"][:, 0] = 1.0
    st["F1"][:, 1] = 1.0
    st["F2"][:, 2] = 1.0
    return st


def jittered_lattice(seed, stream, counts, spacing, origin, jitter):
    """Lattice of counts=(nx,ny,nz) points (x fastest, then z, then y), spacing
    `spacing`, lower corner `origin`, each axis jittered by U(-jitter, +jitter)."""
    nx, ny, nz = counts
    iy, iz, ix = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    p = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float64) * spacing
    p += np.asarray(origin, np.float64)
    n = p.shape[0]
    j = uniform(seed, 3 * n, stream, -jitter, jitter).reshape(n, 3)
    return (p + j).astype(np.float32)


# ----------------------------------------------------------------------------- configs
def elastic_block(seed=1, n_side=20, res=64, substeps=100, dt=1e-4, flip_ratio=-1.0):
    """8,000-particle elastic block: 20^3 lattice, spacing 0.5h, jitter +/-0.25h,
    centre (0.5, 0.7, 0.5) of the unit cube, 64^3 grid, E=1e4 nu=0.3 rho=1,
    gravity -9.8 y, dt=1e-4, APIC."""
    h = 1.0 / res
    sp = 0.5 * h
    half = sp * (n_side - 1) / 2.0
    origin = (0.5 - half, 0.7 - half, 0.5 - half)
    pos = jittered_lattice(seed, 0, (n_side, n_side, n_side), sp, origin, 0.25 * h)
    vp = np.float32(sp) ** 3
    params = StepParams(dt=dt, cell_size=float(np.float32(h)), domain_size=(1.0, 1.0, 1.0), flip_ratio=flip_ratio,
                        materials=[material(MAT_ELASTIC, 1e4, 0.3, 1.0)], forces=[gravity()])
    params.mu_lame, params.lambda_lame = lame(1e4, 0.3)
    params.rho0 = 1.0
    return Scene("elastic_block_8k_64", params, make_state(pos, vp), substeps)


def shear_block(model=MAT_ELASTIC, seed=1, gamma=20.0, substeps=100, dt=1e-4, flip_ratio=-1.0):
    """Parity variant of the elastic block: same 8,000-particle geometry on 64^3,
    rho 1000 instead of 1 (with rho = 1 and E = 1e4 the wave CFL number is
    c dt / h = 0.74 and the reference algorithm blows up within ~40 substeps in
    float32 and float64 alike), and an initial shear velocity v_x = gamma (y - 0.7)
    so that F develops distinct singular values.  model: ELASTIC (E=1e4),
    VON_MISES (E=1e4, q_max=200), DRUCKER_PRAGER (E=3.5e5, rho 1600, 30 deg),
    or the reference's presets for GRANULAR_POWDER, FLUID and VISCOPLASTIC_MUD,
    or FIXED_COROTATED (E=1e4)."""
    sc = elastic_block(seed=seed, substeps=substeps, dt=dt, flip_ratio=flip_ratio)
    if model == MAT_DRUCKER_PRAGER:
        m = material(model, 3.5e5, 0.3, 1600.0, M_friction=math.tan(math.radians(30.0)))
    elif model == MAT_VON_MISES:
        m = material(model, 1e4, 0.3, 1000.0, q_max=200.0)
    elif model == MAT_GRANULAR_POWDER:
        m = preset_powder()
    elif model == MAT_FLUID:
        m = preset_water()
    elif model == MAT_VISCOPLASTIC_MUD:
        m = preset_mud()
    elif model == MAT_FIXED_COROTATED:
        m = material(MAT_FIXED_COROTATED, 1e4, 0.3, 1000.0)
    else:
        m = material(MAT_ELASTIC, 1e4, 0.3, 1000.0)
    sc.params.materials = [m]
    sc.params.rho0 = float(m["rho0"])
    P = sc.state["P"]
    sc.state["v"][:, 0] = (gamma * (P[:, 1].astype(np.float64) - 0.7)).astype(np.float32)
    sc.name = "shear_block_%s_8k_64" % ("elastic", "vonmises", "druckerprager", "powder", "fluid", "mud", "corotated")[model]
    return sc


def multimaterial(seed=2, res=128, substeps=200, dt=5e-5):
    """80,000 particles on 128^3: a 40,000-particle jelly cube (Hencky E=5e3,
    rho 1000) dropped on a 40,000-particle Drucker-Prager sand slab (E=3.5e5,
    friction 30 deg, rho 1600), nu=0.3, APIC, dt=5e-5."""
    h = 1.0 / res
    sp = 0.5 * h
    # jelly: 35^3 lattice truncated to its first 40,000 points (top layer partial)
    jel = jittered_lattice(seed, 0, (35, 35, 35), sp, (0.5 - 17 * sp, 0.35, 0.5 - 17 * sp), 0.25 * h)[:40000]
    # sand slab: 100 x 4 x 100 points resting above the floor band
    sand = jittered_lattice(seed, 1, (100, 4, 100), sp, (0.5 - 49.5 * sp, 3.0 * h, 0.5 - 49.5 * sp), 0.25 * h)
    pos = np.concatenate([jel, sand])
    ids = np.concatenate([np.zeros(40000, np.uint32), np.ones(40000, np.uint32)])
    vp = np.float32(sp) ** 3
    mats = [material(MAT_ELASTIC, 5e3, 0.3, 1000.0),
            material(MAT_DRUCKER_PRAGER, 3.5e5, 0.3, 1600.0, M_friction=math.tan(math.radians(30.0)))]
    params = StepParams(dt=dt, cell_size=float(np.float32(h)), domain_size=(1.0, 1.0, 1.0), flip_ratio=-1.0,
                        materials=mats, forces=[gravity()])
    params.mu_lame, params.lambda_lame = lame(5e3, 0.3)
    return Scene("multimaterial_80k_128", params, make_state(pos, vp, mat_ids=ids), substeps)


def terrain_height(seed, x, z):
    """Synthetic terrain: 0.08 + sum of 8 seeded Gaussian ridges (height 0.05-0.2,
    width 0.05-0.15, each along a seeded line) + one linear channel (depth 0.04)."""
    u = uniform(seed, 8 * 5, 7).reshape(8, 5)
    H = np.full(np.broadcast(x, z).shape, 0.08)
    for i in range(8):
        hgt = 0.05 + 0.15 * u[i, 0]
        wid = 0.05 + 0.10 * u[i, 1]
        cx, cz = u[i, 2], u[i, 3]
        ang = math.pi * u[i, 4]
        d = (x - cx) * math.sin(ang) - (z - cz) * math.cos(ang)
        H = H + hgt * np.exp(-(d / wid) ** 2)
    d = (x - 0.5) * math.sin(0.3) - (z - 0.5) * math.cos(0.3)
    H = H - 0.04 * np.exp(-(d / 0.04) ** 2)
    return H


def terrain_sdf(seed, res, h):
    """Dense Morton-ordered fp32 SDF (sdf[morton(ix,iy,iz)] = y - H(x,z) at cell centres),
    the layout of MPMEngine::setColliderSDF (src/engine/MPMEngine.cpp:204-209)."""
    c = (np.arange(res, dtype=np.float64) + 0.5) * h
    X, Z = np.meshgrid(c, c, indexing="ij")           # [ix, iz]
    H = terrain_height(seed, X, Z)                      # [ix, iz]
    cube = morton_cube_res((res, res, res))
    sdf = np.full(cube ** 3, 1e6, np.float32)
    ix, iy, iz = np.meshgrid(np.arange(res), np.arange(res), np.arange(res), indexing="ij")
    codes = morton_encode(ix.ravel(), iy.ravel(), iz.ravel())
    vals = (c[iy.ravel()] - H[ix.ravel(), iz.ravel()]).astype(np.float32)
    sdf[codes] = vals
    return sdf, H


def slope_flow(seed=3, res=256, n_side=(200, 25, 200), substeps=500, dt=2e-5, with_sdf=True, lift=2.0, vy=0.0):
    """1,000,000 Drucker-Prager particles (friction 35 deg, E=1.4e5, nu=0.3,
    rho 1600) as a jittered slab above a seeded terrain SDF on a 256^3 grid,
    APIC, dt=2e-5.  The slab's lowest layer starts `lift` cells above the
    highest terrain point (2 cells: over the 500 substeps, 0.01 s, it falls
    0.13 cells and never touches the terrain; a negative lift sinks the
    slab's bottom into the ridges), moving at vy (m/s) along y."""
    h = 1.0 / res
    sp = 0.5 * h
    nx, ny, nz = n_side
    ox = 0.5 - sp * (nx - 1) / 2.0
    oz = 0.5 - sp * (nz - 1) / 2.0
    pos = jittered_lattice(seed, 0, (nx, ny, nz), sp, (ox, 0.0, oz), 0.25 * h)
    sdf, H = (terrain_sdf(seed, res, h) if with_sdf else (None, None))
    if H is not None:
        pos[:, 1] += np.float32(H.max() + lift * h)
    else:
        pos[:, 1] += np.float32(0.3)
    vp = np.float32(sp) ** 3
    mats = [material(MAT_DRUCKER_PRAGER, 1.4e5, 0.3, 1600.0, M_friction=math.tan(math.radians(35.0)))]
    params = StepParams(dt=dt, cell_size=float(np.float32(h)), domain_size=(1.0, 1.0, 1.0), flip_ratio=-1.0,
                        materials=mats, forces=[gravity()])
    params.mu_lame, params.lambda_lame = lame(1.4e5, 0.3)
    state = make_state(pos, vp)
    state["v"][:, 1] = np.float32(vy)
    return Scene("slope_flow_1m_256", params, state, substeps, sdf=sdf)


def _mix_shape(u_row, nmin, nmax):
    """Grid resolution and lattice counts of one scene of the mix."""
    n_target = int(round(math.exp(math.log(nmin) + (math.log(nmax) - math.log(nmin)) * u_row[0])))
    res = (64, 96, 128)[min(2, int(u_row[1] * 3))]
    side = max(2, int(round(n_target ** (1.0 / 3.0))))
    ny = max(1, n_target // (side * side))
    return res, (side, ny, side)


def batch_mix_sizes(seed=4, n_scenes=64, nmin=2000, nmax=200000):
    """Particle count of every scene of batch_mix, without building the scenes."""
    u = uniform(seed, n_scenes * 8, 11).reshape(n_scenes, 8)
    out = []
    for s in range(n_scenes):
        _, (nx, ny, nz) = _mix_shape(u[s], nmin, nmax)
        out.append(nx * ny * nz)
    return out


def batch_mix(seed=4, n_scenes=64, substeps=200, dt=1e-4, nmin=2000, nmax=200000, only=None):
    """64 independent scenes: particle counts log-uniform in [2e3, 2e5], grids
    64^3 / 96^3 / 128^3 (unit cube), a jittered box with initial velocity
    U[-1,1]^3, ELASTIC or VON_MISES, and one sphere collider of radius 0.1
    moving with a seeded velocity.  `only` (a set of scene indices) builds a
    subset, e.g. one rank's share."""
    scenes = []
    u = uniform(seed, n_scenes * 8, 11).reshape(n_scenes, 8)
    for s in range(n_scenes):
        if only is not None and s not in only:
            continue
        res, cnt = _mix_shape(u[s], nmin, nmax)
        h = float(np.float32(1.0) / np.float32(res))
        sp = 0.5 * h
        nxz, ny = cnt[0], cnt[1]
        n = nxz * ny * nxz
        ox = 0.5 - sp * (nxz - 1) / 2.0
        oy = 0.45
        pos = jittered_lattice(seed * 1000 + s, 0, cnt, sp, (ox, oy, ox), 0.25 * h)
        vel = uniform(seed * 1000 + s, 3, 1, -1.0, 1.0).astype(np.float32)
        vels = np.broadcast_to(vel, (n, 3)).copy()
        model = MAT_ELASTIC if u[s, 2] < 0.5 else MAT_VON_MISES
        q_max = 50.0 + 450.0 * u[s, 3]
        mats = [material(model, 1e4, 0.3, 1000.0, q_max=q_max)]
        cvel = (uniform(seed * 1000 + s, 3, 2, -0.5, 0.5)).astype(np.float32)
        col = sphere_collider((0.5, 0.25, 0.5), 0.1, vel=tuple(cvel))
        params = StepParams(dt=dt, cell_size=h, domain_size=(1.0, 1.0, 1.0), flip_ratio=-1.0,
                            materials=mats, forces=[gravity()], colliders=[col])
        params.mu_lame, params.lambda_lame = lame(1e4, 0.3)
        scenes.append(Scene("batch_%02d" % s, params, make_state(pos, np.float32(sp) ** 3, vel=vels), substeps))
    return scenes


def collider_track(scene, substeps, start=0):
    """The scene's colliders over `substeps` substeps from substep `start`: each
    moves with its own velocity, pos(k) = pos + vel * (start + k) * dt.
    Returns a (substeps, colliders) record array (one set per substep)."""
    cols = scene.params.colliders_array()[: len(scene.params.colliders)]
    k = (np.arange(substeps, dtype=np.float64) + start) * np.float64(np.float32(scene.params.dt))
    out = np.repeat(cols[None, :], substeps, axis=0)
    out["pos"] = (cols["pos"][None, :, :].astype(np.float64) + k[:, None, None] * cols["vel"][None, :, :]).astype(np.float32)
    return out


def diff_block(seed=5, n=50000, res=64, substeps=200, dt=1e-4, side=37, y0_cells=3.0, vy=-2.0):
    """50,000-particle elastic block for the adjoint: a 37x37x37 lattice (spacing
    0.5h, jitter +/-0.25h) truncated to n points, its base y0_cells cells above
    the floor and falling at vy, so it reaches the wall band and is compressed
    there for the last ~60% of the rollout (with no contact the COM loss would
    not depend on E at all: internal forces conserve momentum).  Per-particle E
    log-uniform in [5e3, 5e4], nu = 0.3, rho0 = 1000, initial velocity
    (0.3, vy, -0.2) + U(+/-0.05), APIC, dt = 1e-4; target point seeded."""
    h = 1.0 / res
    sp = 0.5 * h
    half = (side - 1) / 2.0
    pos = jittered_lattice(seed, 0, (side, side, side), sp, (0.5 - half * sp, y0_cells * h, 0.5 - half * sp), 0.25 * h)[:n]
    n = pos.shape[0]
    noise = uniform(seed, 3 * n, 1, -0.05, 0.05).reshape(n, 3)
    vel = (np.array([0.3, vy, -0.2]) + noise).astype(np.float32)
    E = np.exp(uniform(seed, n, 2, math.log(5e3), math.log(5e4))).astype(np.float32)
    target = (np.array([0.5, 0.3, 0.5]) + uniform(seed, 3, 3, -0.05, 0.05)).astype(np.float32)
    params = StepParams(dt=dt, cell_size=float(np.float32(h)), domain_size=(1.0, 1.0, 1.0), flip_ratio=-1.0,
                        materials=[material(MAT_ELASTIC, 1e4, 0.3, 1000.0)], forces=[gravity()])
    params.mu_lame, params.lambda_lame = lame(1e4, 0.3)
    sc = Scene("diff_block_50k_64", params, make_state(pos, np.float32(sp) ** 3, vel=vel), substeps)
    sc.extra = {"E": E, "nu": 0.3, "rho0": 1000.0, "target": target, "checkpoint_every": 20}
    return sc

# ----------------------------------------------------------------------------- named configurations
CONFIGS_JSON = __import__("pathlib").Path(__file__).with_name("configs.json")


def load_config(key: str):
    """The scene (or, for the batched mix, the list of scenes) of configuration
    `key` in configs.json, built with the seeds and sizes stored there."""
    import json
    cfg = json.loads(CONFIGS_JSON.read_text())["configs"][key]
    args = dict(cfg["args"])
    if "n_side" in args and isinstance(args["n_side"], list):
        args["n_side"] = tuple(args["n_side"])
    return globals()[cfg["generator"]](**args)
