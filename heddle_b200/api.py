"""Host-side mirror of the reference's force / constraint / integrator plugin
surface over the C ABI.

  * PotentialRegistry -- builders keyed by label in the reference's canonical
    order (LJ, SPME real, SPME reciprocal; src/forces/mod.rs:277-289), with
    compositional activation driven by which sections a configuration holds
    and the reference's validation errors (src/forces/mod.rs:394-447);
  * ConstraintRegistry -- "settle" and "shake" groups
    (src/integrator/constraint.rs:205-212, :227-300);
  * IntegratorRegistry -- "velocity-verlet" (with a "lossless" flag) and
    "langevin-baoab" (src/integrator/mod.rs:627-677).

Objects wrap the opaque C handles and raise HeddleError with the library's
status on failure.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from . import units as U
from .systems import SystemSpec


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


class Context:
    """A device, its streams and loaded kernels (init_device,
    src/gpu/device.rs:67-74)."""

    def __init__(self, device: int = 0):
        self.lib = N.load()
        h = C.c_void_p()
        N.check(self.lib.hb_context_create(device, C.byref(h)))
        self.h = h

    def synchronize(self) -> None:
        N.check(self.lib.hb_context_synchronize(self.h))

    def timing(self, enable: bool) -> None:
        N.check(self.lib.hb_timing_enable(self.h, 1 if enable else 0))

    def timings(self) -> np.ndarray:
        out = np.zeros(8)
        N.check(self.lib.hb_timing_get(self.h, N.dptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_context_destroy(self.h)
            self.h = None


class System:
    """Device-resident particle state (ParticleBuffers + SimulationBox)."""

    def __init__(self, ctx: Context, positions, masses, charges, types, box,
                 velocities=None, images=None):
        self.ctx = ctx
        self.lib = ctx.lib
        self._pos = _f64(positions).reshape(-1)
        self._vel = None if velocities is None else _f64(velocities).reshape(-1)
        self._m = _f64(masses)
        self._q = _f64(charges)
        self._t = _u32(types)
        self._img = None if images is None else np.ascontiguousarray(np.asarray(images, dtype=np.int32)).reshape(-1)
        self.n = int(self._m.shape[0])
        d = N.SystemDesc()
        d.n_atoms = self.n
        d.positions = N.dptr(self._pos)
        d.velocities = N.dptr(self._vel)
        d.masses = N.dptr(self._m)
        d.charges = N.dptr(self._q)
        d.types = N.u32ptr(self._t)
        d.images = N.i32ptr(self._img)
        for k in range(6):
            d.box[k] = float(box[k])
        h = C.c_void_p()
        N.check(self.lib.hb_system_create(ctx.h, C.byref(d), C.byref(h)))
        self.h = h

    @classmethod
    def from_spec(cls, ctx: Context, spec: SystemSpec) -> "System":
        return cls(ctx, spec.positions, spec.masses, spec.charges, spec.types, spec.box,
                   velocities=spec.velocities)

    def state(self, out=None):
        """(positions, velocities, images, forces) as (n, 3) arrays; out: four
        C-contiguous arrays to fill instead (float64, float64, int32, float64;
        page-locked ones make the copies fastest)."""
        if out is None:
            out = (np.zeros((self.n, 3)), np.zeros((self.n, 3)), np.zeros((self.n, 3), dtype=np.int32),
                   np.zeros((self.n, 3)))
        pos, vel, img, frc = out
        for a, dt in ((pos, np.float64), (vel, np.float64), (img, np.int32), (frc, np.float64)):
            if a.dtype != dt or not a.flags["C_CONTIGUOUS"] or a.size != 3 * self.n:
                raise ValueError("state(out=...): four C-contiguous (n, 3) arrays of the right types")
        N.check(self.lib.hb_system_get_state(self.h, N.dptr(pos), N.dptr(vel), N.i32ptr(img), N.dptr(frc)))
        return pos.reshape(-1, 3), vel.reshape(-1, 3), img.reshape(-1, 3), frc.reshape(-1, 3)

    def state_f32(self, out):
        """Download into four C-contiguous (n, 3) arrays (float32, float32,
        int32, float32): the single-precision exchange, half the bytes of
        state()."""
        pos, vel, img, frc = out
        for a, dt in ((pos, np.float32), (vel, np.float32), (img, np.int32), (frc, np.float32)):
            if a.dtype != dt or not a.flags["C_CONTIGUOUS"] or a.size != 3 * self.n:
                raise ValueError("state_f32(out=...): four C-contiguous (n, 3) arrays of the right types")
        N.check(self.lib.hb_system_get_state_f32(self.h, N.f32ptr(pos), N.f32ptr(vel), N.i32ptr(img),
                                                 N.f32ptr(frc)))
        return out

    def set_state_f32(self, positions=None, velocities=None) -> None:
        """Upload C-contiguous float32 (n, 3) arrays (None = keep)."""
        for a in (positions, velocities):
            if a is not None and (a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"] or a.size != 3 * self.n):
                raise ValueError("set_state_f32: C-contiguous float32 (n, 3) arrays")
        N.check(self.lib.hb_system_set_state_f32(self.h, N.f32ptr(positions), N.f32ptr(velocities)))

    def positions(self) -> np.ndarray:
        pos = np.zeros(3 * self.n)
        N.check(self.lib.hb_system_get_state(self.h, N.dptr(pos), None, None, None))
        return pos.reshape(-1, 3)

    def forces(self) -> np.ndarray:
        f = np.zeros(3 * self.n)
        N.check(self.lib.hb_system_get_state(self.h, None, None, None, N.dptr(f)))
        return f.reshape(-1, 3)

    def set_state(self, positions=None, velocities=None) -> None:
        p = None if positions is None else _f64(positions).reshape(-1)
        v = None if velocities is None else _f64(velocities).reshape(-1)
        N.check(self.lib.hb_system_set_state(self.h, N.dptr(p), N.dptr(v)))

    def set_box(self, box) -> None:
        b = _f64(box)
        N.check(self.lib.hb_system_set_box(self.h, N.dptr(b)))

    def flip_velocities(self) -> None:
        N.check(self.lib.hb_system_flip_velocities(self.h))

    def box(self) -> np.ndarray:
        b = np.zeros(6)
        N.check(self.lib.hb_system_get_box(self.h, N.dptr(b)))
        return b

    def kinetic(self) -> np.ndarray:
        out = np.zeros(4)
        N.check(self.lib.hb_reduce_kinetic(self.h, N.dptr(out)))
        return out

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_system_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# potentials and their registry
# ---------------------------------------------------------------------------
@dataclass
class LennardJonesParams:
    sigma: np.ndarray
    epsilon: np.ndarray
    cutoff: np.ndarray
    switch: np.ndarray


@dataclass
class SpmeParams:
    alpha: float
    r_cut_real: float
    grid: tuple
    spline_order: int = 4
    reciprocal: bool = True


@dataclass
class HarmonicBondParams:
    atoms: np.ndarray      # [n, 2]
    k: np.ndarray          # hartree / bohr^2
    r0: np.ndarray         # bohr


@dataclass
class HarmonicAngleParams:
    atoms: np.ndarray      # [n, 3], vertex in the middle
    k: np.ndarray          # hartree / rad^2
    theta0: np.ndarray     # rad


@dataclass
class PeriodicDihedralParams:
    atoms: np.ndarray      # [n, 4]
    k: np.ndarray          # hartree
    phi0: np.ndarray       # rad
    n: np.ndarray          # multiplicity


class PotentialBuilder:
    label = ""

    def build(self, config: dict, desc: N.ForceFieldDesc, keep: list) -> bool:
        raise NotImplementedError


class LennardJonesBuilder(PotentialBuilder):
    label = "lennard_jones"

    def build(self, config, desc, keep):
        p = config.get(self.label)
        if p is None:
            return False
        nt = int(np.asarray(p.sigma).shape[0])
        arrs = [_f64(np.asarray(x).reshape(-1)) for x in (p.sigma, p.epsilon, p.cutoff, p.switch)]
        keep.extend(arrs)
        desc.lj_enabled = 1
        desc.n_types = nt
        desc.lj_sigma, desc.lj_epsilon, desc.lj_cutoff, desc.lj_switch = [N.dptr(a) for a in arrs]
        return True


class SpmeBuilder(PotentialBuilder):
    """SPME real-space erfc slot plus, unless disabled, the reciprocal slot."""

    label = "spme"

    def build(self, config, desc, keep):
        p = config.get(self.label)
        if p is None:
            return False
        desc.coulomb_enabled = 1
        desc.alpha = float(p.alpha)
        desc.r_cut_coulomb = float(p.r_cut_real)
        if p.reciprocal:
            desc.recip_enabled = 1
            for k in range(3):
                desc.grid[k] = int(p.grid[k])
            desc.spline_order = int(p.spline_order)
        return True


class HarmonicBondBuilder(PotentialBuilder):
    label = "harmonic_bond"

    def build(self, config, desc, keep):
        p = config.get(self.label)
        if p is None or len(p.k) == 0:
            return False
        arrs = [_u32(np.asarray(p.atoms).reshape(-1)), _f64(p.k), _f64(p.r0)]
        keep.extend(arrs)
        desc.n_bonds = len(arrs[1])
        desc.bond_atoms, desc.bond_k, desc.bond_r0 = N.u32ptr(arrs[0]), N.dptr(arrs[1]), N.dptr(arrs[2])
        return True


class HarmonicAngleBuilder(PotentialBuilder):
    label = "harmonic_angle"

    def build(self, config, desc, keep):
        p = config.get(self.label)
        if p is None or len(p.k) == 0:
            return False
        arrs = [_u32(np.asarray(p.atoms).reshape(-1)), _f64(p.k), _f64(p.theta0)]
        keep.extend(arrs)
        desc.n_angles = len(arrs[1])
        desc.angle_atoms, desc.angle_k, desc.angle_theta0 = (N.u32ptr(arrs[0]), N.dptr(arrs[1]),
                                                             N.dptr(arrs[2]))
        return True


class PeriodicDihedralBuilder(PotentialBuilder):
    label = "periodic_dihedral"

    def build(self, config, desc, keep):
        p = config.get(self.label)
        if p is None or len(p.k) == 0:
            return False
        arrs = [_u32(np.asarray(p.atoms).reshape(-1)), _f64(p.k), _f64(p.phi0), _u32(p.n)]
        keep.extend(arrs)
        desc.n_dihedrals = len(arrs[1])
        desc.dihedral_atoms, desc.dihedral_k = N.u32ptr(arrs[0]), N.dptr(arrs[1])
        desc.dihedral_phi0, desc.dihedral_n = N.dptr(arrs[2]), N.u32ptr(arrs[3])
        return True


class PotentialRegistry:
    """Builders in canonical order (src/forces/mod.rs:277-289: LJ, SPME,
    harmonic bond, harmonic angle, periodic dihedral); a slot is active when
    its section is present (compositional activation)."""

    def __init__(self):
        self.builders: list[PotentialBuilder] = [
            LennardJonesBuilder(), SpmeBuilder(), HarmonicBondBuilder(), HarmonicAngleBuilder(),
            PeriodicDihedralBuilder()]

    def register(self, builder: PotentialBuilder) -> None:
        if any(b.label == builder.label for b in self.builders):
            raise ValueError(f"duplicate potential label {builder.label!r}")
        self.builders.append(builder)

    def labels(self) -> list[str]:
        return [b.label for b in self.builders]


DEFAULT_POTENTIALS = PotentialRegistry()


class ForceField:
    """ForceField::new / step over the C ABI."""

    def __init__(self, system: System, config: dict, exclusions=None, r_skin: float = 0.0,
                 registry: PotentialRegistry | None = None, exact_pairs: bool = False):
        self.system = system
        self.lib = system.lib
        reg = registry or DEFAULT_POTENTIALS
        unknown = set(config) - set(reg.labels())
        if unknown:
            raise ValueError(f"unknown potential sections: {sorted(unknown)}")
        d = N.ForceFieldDesc()
        self._keep: list = []
        self.active = [b.label for b in reg.builders if b.build(config, d, self._keep)]
        if exclusions is not None:
            off, part, slj, sc = exclusions
            arrs = [_u32(off), _u32(part), _f64(slj), _f64(sc)]
            self._keep.extend(arrs)
            d.excl_offsets, d.excl_partners = N.u32ptr(arrs[0]), N.u32ptr(arrs[1])
            d.excl_lj_scale, d.excl_coulomb_scale = N.dptr(arrs[2]), N.dptr(arrs[3])
        d.r_skin = float(r_skin)
        d.pair_mode = N.HB_PAIRS_EXACT if exact_pairs else N.HB_PAIRS_FAST
        h = C.c_void_p()
        N.check(self.lib.hb_forcefield_create(system.h, C.byref(d), C.byref(h)))
        self.h = h

    @classmethod
    def from_spec(cls, system: System, spec: SystemSpec, r_skin: float | None = None,
                  reciprocal: bool = True, exact_pairs: bool = False) -> "ForceField":
        cfg = {}
        if spec.lj_sigma is not None:
            cfg["lennard_jones"] = LennardJonesParams(spec.lj_sigma, spec.lj_epsilon,
                                                      spec.lj_cutoff, spec.lj_switch)
        if spec.alpha is not None:
            cfg["spme"] = SpmeParams(spec.alpha, spec.r_cut_coul, spec.grid, spec.order,
                                     reciprocal=reciprocal and spec.grid is not None)
        bonded = spec.meta.get("bonded") if spec.meta else None
        if bonded:
            for key in ("harmonic_bond", "harmonic_angle", "periodic_dihedral"):
                if key in bonded:
                    cfg[key] = bonded[key]
        excl = None
        if spec.excl_offsets is not None:
            excl = (spec.excl_offsets, spec.excl_partners, spec.excl_lj, spec.excl_coul)
        return cls(system, cfg, excl, spec.r_skin if r_skin is None else r_skin,
                   exact_pairs=exact_pairs)

    def step(self, scalars: bool = False) -> None:
        N.check(self.lib.hb_forcefield_step(
            self.h, N.HB_FORCES_AND_SCALARS if scalars else N.HB_FORCES_ONLY))

    def pre_step(self, force: bool = False) -> bool:
        r = C.c_int(0)
        N.check(self.lib.hb_forcefield_pre_step(self.h, 1 if force else 0, C.byref(r)))
        return bool(r.value)

    def set_launch(self, pair_blocks_per_sm: int | None = None, nl_slab: int | None = None,
                   pair_chunk: int | None = None, fft_plane: bool | None = None,
                   gather_per_offset: bool | None = None, pair_quota: int | None = None) -> None:
        """Launch shapes (autotuned): resident blocks per SM of the persistent
        pair kernel, its packed entries per work item and work items per
        warp (0: persistent blocks); the whole-plane
        transform pass (where the grid has one) or line passes; the gather
        with one thread per (atom, c offset) or per atom.  nl_slab rebuilds
        the packed list at once into slabs of that many entries per i-tile
        (grown again above 3/4 full; too small raises HB_ERR_NL_OVERFLOW and
        halts the force field until a larger slab is set)."""
        for param, v in ((N.HB_LAUNCH_PAIR_BLOCKS_PER_SM, pair_blocks_per_sm),
                         (N.HB_LAUNCH_PAIR_CHUNK, pair_chunk),
                         (N.HB_LAUNCH_PAIR_QUOTA, pair_quota),
                         (N.HB_LAUNCH_FFT_PLANE, fft_plane),
                         (N.HB_LAUNCH_GATHER_FORM, gather_per_offset),
                         (N.HB_LAUNCH_NL_SLAB, nl_slab)):
            if v is not None:
                N.check(self.lib.hb_forcefield_set_launch(self.h, param, int(v)))

    def capacity(self) -> dict:
        """Packed-list capacity: entries per slab, the most entries of one
        i-tile in the last build, slab reallocations, status word."""
        out = np.zeros(4, dtype=np.uint64)
        N.check(self.lib.hb_neighbor_capacity(self.h, out.ctypes.data_as(N.PU64)))
        return dict(zip(["slab", "max_tile_entries", "reallocations", "status"], [int(x) for x in out]))

    def scalars(self) -> dict:
        out = np.zeros(10)
        N.check(self.lib.hb_forcefield_scalars(self.h, N.dptr(out)))
        keys = ["lj", "coulomb_real", "recip", "self", "potential", "virial_pair",
                "virial_recip", "virial", "bonded", "reserved"]
        return dict(zip(keys, out.tolist()))

    def per_atom(self):
        e = np.zeros(self.system.n)
        w = np.zeros(self.system.n)
        N.check(self.lib.hb_forcefield_get_per_atom(self.h, N.dptr(e), N.dptr(w)))
        return e, w

    def neighbor_pairs(self):
        cnt = C.c_uint64(0)
        dup = C.c_uint64(0)
        N.check(self.lib.hb_neighbor_pairs(self.h, None, 0, C.byref(cnt), C.byref(dup)))
        buf = np.zeros(2 * max(cnt.value, 1), dtype=np.uint32)
        N.check(self.lib.hb_neighbor_pairs(self.h, N.u32ptr(buf), cnt.value, C.byref(cnt), C.byref(dup)))
        return buf[: 2 * cnt.value].reshape(-1, 2), int(dup.value)

    def stats(self) -> dict:
        out = np.zeros(6, dtype=np.uint64)
        N.check(self.lib.hb_neighbor_stats(self.h, out.ctypes.data_as(N.PU64)))
        keys = ["tiles", "entries", "capacity", "rebuilds", "status", "pair_slots"]
        return dict(zip(keys, [int(x) for x in out]))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_forcefield_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# constraints
# ---------------------------------------------------------------------------
CONSTRAINT_KINDS = {"settle": N.HB_CONSTRAINT_SETTLE, "shake": N.HB_CONSTRAINT_SHAKE}


class Constraints:
    """Constraint hooks of SETTLE / SHAKE groups (Constraint trait,
    src/integrator/constraint.rs:43-122)."""

    def __init__(self, system: System, group_offsets, group_atoms, group_kind,
                 settle_geometry=None, shake=None, shake_tol: float = 3.57e-6,
                 shake_max_iter: int = 32, shake_tol_relative: bool = False):
        self.system = system
        self.lib = system.lib
        d = N.ConstraintsDesc()
        go, ga, gk = _u32(group_offsets), _u32(group_atoms), _u32(group_kind)
        self._keep = [go, ga, gk]
        d.n_groups = int(gk.shape[0])
        d.group_offsets, d.group_atoms, d.group_kind = N.u32ptr(go), N.u32ptr(ga), N.u32ptr(gk)
        if settle_geometry is not None:
            ra, rb, rc = [_f64(x) for x in settle_geometry]
            self._keep += [ra, rb, rc]
            d.settle_ra, d.settle_rb, d.settle_rc = N.dptr(ra), N.dptr(rb), N.dptr(rc)
        if shake is not None:
            co, ci, cj, cd = _u32(shake[0]), _u32(shake[1]), _u32(shake[2]), _f64(shake[3])
            self._keep += [co, ci, cj, cd]
            d.con_offsets, d.con_i, d.con_j, d.con_dist = N.u32ptr(co), N.u32ptr(ci), N.u32ptr(cj), N.dptr(cd)
        d.shake_tol = float(shake_tol)
        d.shake_max_iter = int(shake_max_iter)
        d.shake_tol_relative = 1 if shake_tol_relative else 0
        h = C.c_void_p()
        N.check(self.lib.hb_constraints_create(system.h, C.byref(d), C.byref(h)))
        self.h = h
        self._mlp = None

    @classmethod
    def from_spec(cls, system: System, spec: SystemSpec, **kw) -> "Constraints":
        geo = None
        if spec.settle_ra is not None:
            geo = (spec.settle_ra, spec.settle_rb, spec.settle_rc)
        shake = None
        if spec.con_offsets is not None:
            shake = (spec.con_offsets, spec.con_i, spec.con_j, spec.con_dist)
        if "shake_rel_tol" in (spec.meta or {}) and "shake_tol" not in kw:
            kw.setdefault("shake_tol", spec.meta["shake_rel_tol"])
            kw.setdefault("shake_tol_relative", True)
            kw.setdefault("shake_max_iter", 200)
        return cls(system, spec.group_offsets, spec.group_atoms, spec.group_kind, geo, shake, **kw)

    def before_drift(self):
        N.check(self.lib.hb_constraints_before_drift(self.h))

    def after_drift(self, dt: float):
        N.check(self.lib.hb_constraints_after_drift(self.h, float(dt)))

    def after_kick(self, dt: float):
        N.check(self.lib.hb_constraints_after_kick(self.h, float(dt)))

    def virial(self) -> np.ndarray:
        out = np.zeros(self.system.n)
        N.check(self.lib.hb_constraints_get_virial(self.h, N.dptr(out)))
        return out

    def shake_stats(self, reset: bool = False) -> dict:
        out = np.zeros(3)
        N.check(self.lib.hb_constraints_shake_stats(self.h, N.dptr(out), 1 if reset else 0))
        return {"group_sweeps": out[0], "solves": out[1], "mean_sweeps": out[2]}

    def record(self, enable: bool = True) -> None:
        N.check(self.lib.hb_constraints_record(self.h, 1 if enable else 0))

    def fuse_head(self, enable: bool = True) -> None:
        """Langevin steps of an all-SETTLE system: the head (kick, velocity
        projection, drift / O / drift, position reset) as one kernel (True,
        the default) or as four (False); the results are identical."""
        N.check(self.lib.hb_constraints_fuse_head(self.h, 1 if enable else 0))

    def get_record(self) -> dict:
        m = C.c_uint32(0)
        N.check(self.lib.hb_constraints_get_record(self.h, None, None, None, None, C.byref(m)))
        k = m.value
        f = np.zeros(8 * max(k, 1), dtype=np.float32)
        l1, ls, lam = np.zeros(max(k, 1)), np.zeros(max(k, 1)), np.zeros(max(k, 1))
        N.check(self.lib.hb_constraints_get_record(self.h, N.f32ptr(f), N.dptr(l1), N.dptr(ls),
                                                   N.dptr(lam), C.byref(m)))
        return {"features": f[: 8 * k].reshape(k, 8), "lam1": l1[:k], "lscale": ls[:k], "lam": lam[:k]}

    def set_warm_start(self, mlp: "ShakeMLP | None") -> None:
        N.check(self.lib.hb_constraints_set_warm_start(self.h, mlp.h if mlp else None))
        self._mlp = mlp

    def choose_warm_start(self, mlp: "ShakeMLP", ff: "ForceField", kind: str, dt: float,
                          steps: int = 50, **integrator_kw) -> dict:
        """Cost gate of the learned warm start: time `steps` CUDA-graph steps
        with plain SHAKE and with the network's initial multipliers (device
        time, a scratch integrator of the given kind, the state restored
        after each run) and attach the network only if its step is faster --
        the feature pass and the inference cost a fixed time per step, the
        sweeps they save scale with the SHAKE work.  Returns both timings,
        the mean sweeps per group solve, and the choice."""
        sys_ = self.system
        ctx = sys_.ctx
        pos, vel, _, _ = sys_.state()
        box = sys_.box()
        out = {}
        for label, net in (("plain", None), ("learned", mlp)):
            self.set_warm_start(net)
            it = Integrator(sys_, kind, dt, **integrator_kw)
            it.step_graph(ff, self, n_steps=3)
            self.shake_stats(reset=True)
            ctx.timing(True)
            it.step_graph(ff, self, n_steps=steps)
            ms = float(ctx.timings()[0])
            ctx.timing(False)
            st = self.shake_stats()
            it.close()
            sys_.set_box(box)
            sys_.set_state(pos, vel)
            ff.pre_step(force=True)
            out[label] = {"ms_per_step": ms / steps, "mean_sweeps": st["mean_sweeps"]}
        use = out["learned"]["ms_per_step"] < out["plain"]["ms_per_step"]
        self.set_warm_start(mlp if use else None)
        out["chosen"] = "learned" if use else "plain"
        return out

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_constraints_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# integrators
# ---------------------------------------------------------------------------
INTEGRATOR_KINDS = {
    "velocity-verlet": N.HB_INTEGRATOR_VV,
    "velocity-verlet-lossless": N.HB_INTEGRATOR_VV_LOSSLESS,
    "langevin-baoab": N.HB_INTEGRATOR_LANGEVIN,
}


class Integrator:
    def __init__(self, system: System, kind: str, dt: float, friction: float = 0.0,
                 temperature: float = 0.0, seed: int = 0, step0: int = 0):
        if kind not in INTEGRATOR_KINDS:
            raise ValueError(f"unknown integrator {kind!r}; known: {sorted(INTEGRATOR_KINDS)}")
        self.system = system
        self.lib = system.lib
        d = N.IntegratorDesc()
        d.kind = INTEGRATOR_KINDS[kind]
        d.dt = float(dt)
        d.friction = float(friction)
        d.temperature = float(temperature)
        d.seed = int(seed)
        d.step0 = int(step0)
        h = C.c_void_p()
        N.check(self.lib.hb_integrator_create(system.h, C.byref(d), C.byref(h)))
        self.h = h

    def step(self, ff: ForceField, cons: Constraints | None = None, n_steps: int = 1,
             scalar_every: int = 0) -> None:
        N.check(self.lib.hb_integrator_step(self.h, ff.h, cons.h if cons else None,
                                            int(n_steps), int(scalar_every)))

    def step_graph(self, ff: ForceField, cons: Constraints | None = None, n_steps: int = 1) -> None:
        N.check(self.lib.hb_integrator_step_graph(self.h, ff.h, cons.h if cons else None, int(n_steps)))

    def step_exchange(self, ff: ForceField, cons: Constraints | None = None, n_steps: int = 1,
                      positions_in=None, velocities_in=None, out=None):
        """Upload float32 (n, 3) positions / velocities (None = keep), run
        n_steps graph steps and read the state after the last one into
        `out` = (positions, velocities, images, forces) arrays (float32,
        float32, int32, float32; any None).  With page-locked arrays the
        read-out of positions and images overlaps the last step's force
        evaluation."""
        want = ((np.float32, positions_in), (np.float32, velocities_in))
        pos, vel, img, frc = out if out is not None else (None, None, None, None)
        want += ((np.float32, pos), (np.float32, vel), (np.int32, img), (np.float32, frc))
        n = self.system.n
        for dt, a in want:
            if a is not None and (a.dtype != dt or not a.flags["C_CONTIGUOUS"] or a.size != 3 * n):
                raise ValueError("step_exchange: C-contiguous (n, 3) arrays of the right types")
        N.check(self.lib.hb_integrator_step_exchange_f32(
            self.h, ff.h, cons.h if cons else None, int(n_steps), N.f32ptr(positions_in),
            N.f32ptr(velocities_in), N.f32ptr(pos), N.f32ptr(vel), N.i32ptr(img), N.f32ptr(frc)))
        return out

    def count_launches(self, ff: ForceField, cons: Constraints | None = None) -> tuple:
        """(kernels every step, kernels of one neighbour rebuild, kernels of
        one barostat move or 0)."""
        out = np.zeros(3, dtype=np.uint64)
        N.check(self.lib.hb_integrator_count_launches(self.h, ff.h, cons.h if cons else None,
                                                      out.ctypes.data_as(N.PU64)))
        return int(out[0]), int(out[1]), int(out[2])

    def set_barostat(self, baro: "Barostat | PressureCoupling | None") -> None:
        """Attach a Monte-Carlo barostat or a per-step pressure coupling
        (c-rescale, Berendsen); None detaches both."""
        if baro is None:
            N.check(self.lib.hb_integrator_set_barostat(self.h, None))
            N.check(self.lib.hb_integrator_set_pcouple(self.h, None))
        elif isinstance(baro, PressureCoupling):
            N.check(self.lib.hb_integrator_set_pcouple(self.h, baro.h))
        else:
            N.check(self.lib.hb_integrator_set_barostat(self.h, baro.h))
        self._baro = baro

    def set_thermostat(self, thermo: "Thermostat | None") -> None:
        """Attach (or detach with None) a velocity thermostat (CSVR,
        Andersen, Berendsen); velocity Verlet only."""
        N.check(self.lib.hb_integrator_set_thermostat(self.h, thermo.h if thermo else None))
        self._thermo = thermo

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_integrator_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# barostats (registry kind names of src/integrator/mc_barostat.rs:371-379)
# ---------------------------------------------------------------------------
BAROSTAT_STATS = ("volume", "acceptance", "max_volume_step", "conserved_term", "attempted",
                  "accepted", "last_dv", "last_w", "last_u_old", "last_u_new", "last_scale",
                  "last_accepted", "last_trial", "last_u2", "draws")


class Barostat:
    """Monte-Carlo barostat ("monte-carlo"): a device-side Metropolis volume
    move on molecular centres of mass every `frequency` steps.  pressure in
    hartree/bohr^3, temperature as k_B T in hartree, volume_step in bohr^3
    (None: 1 % of the initial volume).  molecules = (offsets, atoms) CSR
    covering every atom once; None makes every atom its own molecule."""

    kind = "monte-carlo"

    def __init__(self, system: System, pressure: float, temperature: float, seed: int,
                 frequency: int = 25, volume_step: float | None = None, molecules=None):
        self.system = system
        self.lib = system.lib
        d = N.BarostatDesc()
        d.pressure = float(pressure)
        d.temperature = float(temperature)
        d.frequency = int(frequency)
        d.volume_step = float(volume_step) if volume_step is not None else 0.0
        d.seed = int(seed)
        self._keep = []
        if molecules is not None:
            off = np.ascontiguousarray(molecules[0], dtype=np.uint32)
            atoms = np.ascontiguousarray(molecules[1], dtype=np.uint32)
            self._keep += [off, atoms]
            d.n_molecules = len(off) - 1
            d.mol_offsets = N.u32ptr(off)
            d.mol_atoms = N.u32ptr(atoms)
        h = C.c_void_p()
        N.check(self.lib.hb_barostat_create(system.h, C.byref(d), C.byref(h)))
        self.h = h

    def move(self, ff: ForceField) -> None:
        """One Barostat::apply_move; ff's last evaluation must carry scalars."""
        N.check(self.lib.hb_barostat_mc_move(self.h, ff.h))

    def stats(self) -> dict:
        out = np.zeros(len(BAROSTAT_STATS))
        N.check(self.lib.hb_barostat_stats(self.h, N.dptr(out)))
        return dict(zip(BAROSTAT_STATS, out.tolist()))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_barostat_destroy(self.h)
            self.h = None


MIN_REASONS = {1: "force_tolerance", 2: "energy_tolerance", 3: "force_zero"}


class Minimizer:
    """Steepest-descent minimisation ("steepest-descent") of ff's energy with
    cons' groups projected after every trial step; lengths in bohr, forces
    in hartree/bohr, energy_tolerance relative.  Defaults are the
    reference's (initial_step 1e-12 m, max_step 1e-10 m, x1.2 / x0.2,
    force_tolerance 1e-10 N, energy_tolerance 1e-7, 1000 iterations)."""

    def __init__(self, ff: ForceField, cons: "Constraints | None" = None,
                 initial_step: float = 1.0e-12 / U.BOHR_M,
                 max_step: float = 1.0e-10 / U.BOHR_M, step_increase: float = 1.2,
                 step_decrease: float = 0.2, force_tolerance: float = 1.0e-10 / U.FORCE_N,
                 energy_tolerance: float = 1.0e-7, max_iterations: int = 1000):
        self.ff = ff
        self.lib = ff.lib
        d = N.MinimizerDesc()
        d.initial_step = float(initial_step)
        d.max_step = float(max_step)
        d.step_increase = float(step_increase)
        d.step_decrease = float(step_decrease)
        d.force_tolerance = float(force_tolerance)
        d.energy_tolerance = float(energy_tolerance)
        d.max_iterations = int(max_iterations)
        self.max_iterations = int(max_iterations)
        h = C.c_void_p()
        N.check(self.lib.hb_minimizer_create(ff.h, cons.h if cons else None, C.byref(d), C.byref(h)))
        self.h = h

    @staticmethod
    def _row(r) -> dict:
        return {"iteration": int(r.iteration), "energy": r.energy, "max_force": r.max_force,
                "step": r.step, "accepted": bool(r.accepted),
                "converged": MIN_REASONS.get(int(r.converged))}

    def begin(self) -> dict:
        """Forces and energy at the current positions: the iteration-0 report."""
        r = N.MinReport()
        N.check(self.lib.hb_minimizer_begin(self.h, C.byref(r)))
        return self._row(r)

    def iterate(self, n: int) -> list:
        """Up to n iterations (fewer at convergence or max_iterations)."""
        buf = (N.MinReport * max(int(n), 1))()
        done = C.c_uint32(0)
        N.check(self.lib.hb_minimizer_iterate(self.h, int(n), buf, C.byref(done)))
        return [self._row(buf[k]) for k in range(done.value)]

    def run(self, chunk: int = 64) -> list:
        """begin() then iterations until convergence or max_iterations; all reports."""
        out = [self.begin()]
        while out[-1]["converged"] is None and out[-1]["iteration"] < self.max_iterations:
            rows = self.iterate(chunk)
            if not rows:
                break
            out += rows
        return out

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_minimizer_destroy(self.h)
            self.h = None


THERMOSTAT_KINDS = {"csvr": 0, "andersen": 1, "berendsen": 2}
THERMOSTAT_STATS = ("injection", "kinetic", "factor", "sum_squares", "r", "draws", "dof")


class Thermostat:
    """Velocity thermostat for velocity Verlet, applied after each step's
    constraint velocity projection (the reference's post-force slot):
    "csvr" (Bussi stochastic velocity rescaling, tau), "andersen"
    (per-atom Maxwell-Boltzmann collisions at collision_rate) or
    "berendsen" (weak coupling, tau).  temperature as k_B T in hartree,
    times in a.u.; n_constraints is removed from the degrees of freedom."""

    def __init__(self, system: System, kind: str, temperature: float, seed: int = 0,
                 tau: float = 0.0, collision_rate: float = 0.0, n_constraints: int = 0):
        if kind not in THERMOSTAT_KINDS:
            raise ValueError(f"unknown thermostat kind {kind!r}")
        self.system = system
        self.lib = system.lib
        self.kind = kind
        d = N.ThermostatDesc()
        d.kind = THERMOSTAT_KINDS[kind]
        d.temperature = float(temperature)
        d.tau = float(tau)
        d.collision_rate = float(collision_rate)
        d.seed = int(seed)
        d.n_constraints = int(n_constraints)
        h = C.c_void_p()
        N.check(self.lib.hb_thermostat_create(system.h, C.byref(d), C.byref(h)))
        self.h = h

    def stats(self) -> dict:
        out = np.zeros(len(THERMOSTAT_STATS))
        N.check(self.lib.hb_thermostat_stats(self.h, N.dptr(out)))
        return dict(zip(THERMOSTAT_STATS, out.tolist()))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_thermostat_destroy(self.h)
            self.h = None


PCOUPLE_KINDS = {"c_rescale": 0, "berendsen": 1}
PCOUPLE_STATS = ("pressure", "volume", "injection", "mu", "draws", "kinetic", "virial", "guarded")


class PressureCoupling:
    """Per-step isotropic pressure coupling for velocity Verlet: "c_rescale"
    (stochastic cell rescaling) or "berendsen".  pressure in hartree/bohr^3,
    temperature as k_B T in hartree, tau in a.u., compressibility in
    bohr^3/hartree."""

    def __init__(self, system: System, kind: str, pressure: float, tau: float,
                 compressibility: float, temperature: float = 0.0, seed: int = 0):
        if kind not in PCOUPLE_KINDS:
            raise ValueError(f"unknown pressure coupling kind {kind!r}")
        self.system = system
        self.lib = system.lib
        self.kind = kind
        d = N.PcoupleDesc()
        d.kind = PCOUPLE_KINDS[kind]
        d.pressure = float(pressure)
        d.temperature = float(temperature)
        d.tau = float(tau)
        d.compressibility = float(compressibility)
        d.seed = int(seed)
        h = C.c_void_p()
        N.check(self.lib.hb_pcouple_create(system.h, C.byref(d), C.byref(h)))
        self.h = h

    def stats(self) -> dict:
        out = np.zeros(len(PCOUPLE_STATS))
        N.check(self.lib.hb_pcouple_stats(self.h, N.dptr(out)))
        return dict(zip(PCOUPLE_STATS, out.tolist()))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_pcouple_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# batched replicas
# ---------------------------------------------------------------------------
class Batch:
    """Independent systems advanced together: every member's step in one
    CUDA graph (one parallel branch per member context), one graph launch
    per step.  members: list of (Integrator, ForceField, Constraints | None),
    each on a Context of its own; ctx launches the graph."""

    def __init__(self, ctx: Context, members):
        self.ctx = ctx
        self.lib = ctx.lib
        self.members = list(members)
        n = len(self.members)
        arr = C.c_void_p * n
        its = arr(*[m[0].h for m in self.members])
        ffs = arr(*[m[1].h for m in self.members])
        cons = arr(*[(m[2].h if m[2] is not None else None) for m in self.members])
        h = C.c_void_p()
        N.check(self.lib.hb_batch_create(ctx.h, n, its, ffs, cons, C.byref(h)))
        self.h = h

    def step(self, n_steps: int = 1) -> None:
        N.check(self.lib.hb_batch_step(self.h, int(n_steps)))

    def set_pair_form(self, one_launch: bool) -> None:
        """One multi-system pair kernel for all members (when they share the
        pair physics) or one pair kernel per member (default, faster)."""
        N.check(self.lib.hb_batch_set_pair_form(self.h, 1 if one_launch else 0))

    def pair_form(self) -> bool:
        v = C.c_int(0)
        N.check(self.lib.hb_batch_pair_form(self.h, C.byref(v)))
        return bool(v.value)

    def count_launches(self) -> tuple:
        out = np.zeros(2, dtype=np.uint64)
        N.check(self.lib.hb_batch_count_launches(self.h, out.ctypes.data_as(N.PU64)))
        return int(out[0]), int(out[1])

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_batch_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------------------
# learned SHAKE warm start
# ---------------------------------------------------------------------------
class ShakeMLP:
    """8 -> 64 -> 64 -> 1 tanh network whose hidden layers run as BF16
    tensor-core GEMMs (forward, backward, Adam training on the device)."""

    N_FEATURES = 8

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        N.check(self.lib.hb_shake_mlp_create(ctx.h, int(seed), C.byref(h)))
        self.h = h
        self.n_params = int(self.lib.hb_shake_mlp_param_count())

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        N.check(self.lib.hb_shake_mlp_get_params(self.h, N.f32ptr(out), self.n_params))
        return out

    def set_params(self, p) -> None:
        a = np.ascontiguousarray(p, dtype=np.float32)
        N.check(self.lib.hb_shake_mlp_set_params(self.h, N.f32ptr(a), self.n_params))

    def set_normalization(self, mean, inv_std, target_scale: float) -> None:
        m = np.ascontiguousarray(mean, dtype=np.float32)
        s = np.ascontiguousarray(inv_std, dtype=np.float32)
        N.check(self.lib.hb_shake_mlp_set_normalization(self.h, N.f32ptr(m), N.f32ptr(s),
                                                        float(target_scale)))

    def set_wait_limit(self, polls: int = 1 << 22, issue: bool = True) -> None:
        """Poll limit of the network kernels' bounded waits; issue=False makes
        the next inference issue no tensor-core work, so its wait runs out
        (HB_ERR_DEVICE_TIMEOUT, the failure-path test)."""
        N.check(self.lib.hb_shake_mlp_set_wait_limit(self.h, int(polls), 1 if issue else 0))

    def predict(self, features) -> np.ndarray:
        f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1)
        n = f.size // self.N_FEATURES
        out = np.zeros(max(n, 1), dtype=np.float32)
        N.check(self.lib.hb_shake_mlp_predict(self.h, N.f32ptr(f), n, N.f32ptr(out)))
        return out[:n]

    def gradients(self, features, targets):
        f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_double(0.0)
        N.check(self.lib.hb_shake_mlp_gradients(self.h, N.f32ptr(f), N.f32ptr(t), t.size,
                                                N.f32ptr(g), C.byref(loss)))
        return g, loss.value

    def train(self, features, targets, epochs: int, batch: int = 512, lr: float = 1e-3,
              seed: int = 0) -> np.ndarray:
        f = np.ascontiguousarray(features, dtype=np.float32).reshape(-1)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        losses = np.zeros(epochs)
        N.check(self.lib.hb_shake_mlp_train(self.h, N.f32ptr(f), N.f32ptr(t), t.size, int(epochs),
                                            int(batch), float(lr), int(seed), N.dptr(losses)))
        return losses

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.hb_shake_mlp_destroy(self.h)
            self.h = None
