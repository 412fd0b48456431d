"""koral_b200: B200 (sm_100a) implementation of KORAL's per-step hot path.

The package is a thin host-side mirror of KORAL's own operator interface
(op_explicit, op_implicit, calc_u2p, set_bc, copyi_u, addi_u, save_timesteps,
finite.c) over the C-ABI library ``_lib/libkoral_b200.so`` declared in
``include/koral_b200.h``.  Arrays cross the boundary in KORAL's layout
(cell-major, variable fastest, ghost cells included: ``[SZ][SY][SX][NV]``).

There is no CPU fallback: if the CUDA library is missing or no GPU is
visible, constructing a ``Subdomain`` raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("KORAL_B200_LIB") or os.path.join(HERE, "_lib", "libkoral_b200.so")

PPM, MP5 = 2, 4
BC_PERIODIC, BC_OUTFLOW, BC_REFLECT, BC_PERIODIC_COPY = 0, 1, 2, 3
LAXF, HLL = 0, 1
ARR_U, ARR_P, ARR_UT0, ARR_UT1, ARR_UT2 = 0, 1, 2, 3, 4
POLAR_CORRECT, POLAR_CORRECT_3D, POLAR_SMOOTH = 1, 2, 4   # KGPU_POLAR_* (kgpu_set_polar_correction)

_dp = ctypes.POINTER(ctypes.c_double)


class RadParams(ctypes.Structure):
    """kgpu_rad_params (include/koral_b200.h)."""
    _fields_ = [(n, ctypes.c_double) for n in (
        "gamma", "kb", "mp", "sigma", "mu", "ggg", "ccc", "masscm", "kramers", "kes", "kes_gu", "gammamaxrad",
        "eradfloor", "gammasmalllimit", "numepsilon", "eps", "conv", "entrconv", "maxiter", "dampfac", "maxdown",
        "maxup", "maxdamping", "threshold", "u2pconv", "eerhoratiomin", "eerhoratiomax", "eeuuratiomin",
        "eeuuratiomax")]


class SolverOpts(ctypes.Structure):
    """kgpu_rad_solver_opts (include/koral_b200.h): tuning of the batched and
    persistent implicit solvers."""
    _fields_ = [(n, ctypes.c_int) for n in ("pass_iters", "inner_cap", "tail", "warm_attempts", "thin",
                                            "blocks_per_sm", "skip", "hard")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class Tuning(ctypes.Structure):
    """kgpu_tuning (include/koral_b200.h): launch shapes and solver settings
    of a context."""
    _fields_ = [("flux_blocks", ctypes.c_int), ("flux_split", ctypes.c_int), ("update_blocks", ctypes.c_int),
                ("u2p_blocks", ctypes.c_int),
                ("u2p_pass_iters", ctypes.c_int), ("implicit_mode", ctypes.c_int), ("implicit", SolverOpts)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_ if n != "implicit"}
        d["implicit"] = self.implicit.as_dict()
        return d


class ScalarsParams(ctypes.Structure):
    _fields_ = [("spin", ctypes.c_double), ("mass", ctypes.c_double), ("bhdisk", ctypes.c_int)]


NSCALARS = 13


class KgpuError(RuntimeError):
    pass


class Config(ctypes.Structure):
    """kgpu_config of include/koral_b200.h."""

    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("ng", ctypes.c_int), ("nv", ctypes.c_int),
        ("int_order", ctypes.c_int), ("fluxmethod", ctypes.c_int),
        ("axisym_metric", ctypes.c_int), ("bc", ctypes.c_int * 3),
        ("gamma", ctypes.c_double), ("tsteplim", ctypes.c_double),
        ("rhofloor", ctypes.c_double), ("uurhoratiomin", ctypes.c_double),
        ("uurhoratiomax", ctypes.c_double), ("b2rhoratiomax", ctypes.c_double),
        ("gammamaxhd", ctypes.c_double), ("u2pconv", ctypes.c_double),
    ]


class TorusParams(ctypes.Structure):
    """kgpu_torus_params of include/koral_b200.h."""

    _fields_ = [
        ("spin", ctypes.c_double), ("r0", ctypes.c_double), ("h0", ctypes.c_double),
        ("r_lo", ctypes.c_double), ("r_hi", ctypes.c_double),
        ("x2_lo", ctypes.c_double), ("x2_hi", ctypes.c_double),
        ("rin", ctypes.c_double), ("rmax", ctypes.c_double), ("kappa", ctypes.c_double),
        ("noise", ctypes.c_double), ("seed", ctypes.c_ulonglong),
        ("atm_rho0", ctypes.c_double), ("atm_uu0", ctypes.c_double), ("maxbeta", ctypes.c_double),
    ]


_LIB = None


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise KgpuError(f"{LIB_PATH} is missing: build it with koral_b200.build.build()")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        sig = {
            "kgpu_default_config": [ctypes.POINTER(Config), ctypes.c_int, ctypes.c_int, ctypes.c_int],
            "kgpu_create": [ctypes.POINTER(Config), ctypes.POINTER(vp)],
            "kgpu_destroy": [vp],
            "kgpu_upload_grid": [vp, _dp, _dp, _dp],
            "kgpu_set_uniform_grid": [vp, _dp, _dp],
            "kgpu_upload_metric": [vp] + [_dp] * 9,
            "kgpu_set_minkowski_metric": [vp],
            "kgpu_set_density_floor": [vp, _dp, _dp],
            "kgpu_upload_state": [vp, _dp, _dp],
            "kgpu_download_state": [vp, _dp, _dp],
            "kgpu_download_array": [vp, ctypes.c_int, _dp],
            "kgpu_op_explicit": [vp, ctypes.c_double, ctypes.c_double],
            "kgpu_op_implicit": [vp, ctypes.c_double, ctypes.c_double],
            "kgpu_calc_u2p": [vp],
            "kgpu_set_bc": [vp, ctypes.c_double, ctypes.c_int],
            "kgpu_save_timesteps": [vp],
            "kgpu_copyi_u": [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int],
            "kgpu_addi_u": [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int],
            "kgpu_begin_run": [vp],
            "kgpu_begin_step": [vp, _dp],
            "kgpu_get_tstepdenmax": [vp, _dp],
            "kgpu_set_tstepdenmax": [vp, ctypes.c_double],
            "kgpu_rk2_steps": [vp, ctypes.c_int],
            "kgpu_rk2_steps_graph": [vp, ctypes.c_int],
            "kgpu_get_counters": [vp, ctypes.POINTER(ctypes.c_ulonglong)],
            "kgpu_reset_counters": [vp],
            "kgpu_get_counters_ex": [vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int],
            "kgpu_set_u2p_pass_iters": [vp, ctypes.c_int],
            "kgpu_init_orszag_tang": [vp],
            "kgpu_u2p_cells": [ctypes.c_int, ctypes.POINTER(Config), _dp, _dp, _dp, _dp,
                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
            "kgpu_p2u_cells": [ctypes.c_int, ctypes.POINTER(Config), _dp, _dp, _dp, _dp],
            "kgpu_default_torus_params": [ctypes.POINTER(TorusParams)],
            "kgpu_mks2_metric_tables": [ctypes.c_double] * 3 + [ctypes.c_int] * 5 + [_dp] * 12,
            "kgpu_fm_torus_state": [ctypes.POINTER(TorusParams), ctypes.POINTER(Config)] + [_dp] * 7,
            "kgpu_fm_torus_floor": [ctypes.POINTER(TorusParams), ctypes.c_int, ctypes.c_int, _dp, _dp, _dp],
            "kgpu_init_fm_torus": [vp, ctypes.POINTER(TorusParams)],
            "kgpu_init_fm_torus_host": [vp, ctypes.POINTER(TorusParams)],
            "kgpu_download_metric": [vp] + [_dp] * 9,
            "kgpu_calc_scalars": [vp, ctypes.POINTER(ScalarsParams), ctypes.c_double, _dp],
            "kgpu_calc_scalars_device": [vp, ctypes.POINTER(ScalarsParams), ctypes.c_double, vp],
            "kgpu_download_flux": [vp, ctypes.c_int, _dp],
            "kgpu_write_restart": [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int],
            "kgpu_read_restart": [vp, ctypes.c_char_p, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int)],
            "kgpu_download_emf": [vp, _dp],
            "kgpu_set_polar_correction": [vp, ctypes.c_int, ctypes.c_int],
            "kgpu_avg_count": [vp],
            "kgpu_set_avg": [vp, ctypes.c_int, ctypes.c_double],
            "kgpu_save_avg": [vp, ctypes.c_double],
            "kgpu_download_avg": [vp, _dp, _dp],
            "kgpu_reset_avg": [vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.kgpu_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.kgpu_profile_enable.argtypes = [vp, ctypes.c_int]
        L.kgpu_profile_read.argtypes = [vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(ctypes.c_char_p)]
        L.kgpu_profile_reset.argtypes = [vp]
        L.kgpu_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.kgpu_last_error.restype = ctypes.c_char_p
        ip_ = ctypes.POINTER(ctypes.c_int)
        rpp = ctypes.POINTER(RadParams)
        L.kgpu_rad_default_params.argtypes = [rpp] + [ctypes.c_double] * 4
        L.kgpu_rad_implicit_cells.argtypes = [ctypes.c_int, rpp] + [_dp] * 7 + [ip_] * 3 + [ctypes.c_int]
        L.kgpu_rad_implicit_cells_device.argtypes = [ctypes.c_int, rpp] + [vp] * 10 + [ctypes.c_int, vp, vp,
                                                     ctypes.POINTER(ctypes.c_ulonglong)]
        L.kgpu_rad_work_bytes.argtypes = [ctypes.c_int]
        L.kgpu_rad_work_bytes.restype = ctypes.c_size_t
        L.kgpu_rad_u2p_cells.argtypes = [ctypes.c_int, rpp] + [_dp] * 4 + [ip_] * 2
        L.kgpu_rad_p2u_cells.argtypes = [ctypes.c_int, rpp] + [_dp] * 4
        L.kgpu_rad_set_pass_iters.argtypes = [ctypes.c_int]
        L.kgpu_rad_set_inner_cap.argtypes = [ctypes.c_int]
        L.kgpu_rad_set_tail.argtypes = [ctypes.c_int]
        L.kgpu_rad_set_warm_attempts.argtypes = [ctypes.c_int]
        L.kgpu_ks_metric.argtypes = [ctypes.c_double] * 3 + [_dp] * 2
        L.kgpu_ks_metric_batch.argtypes = [ctypes.c_double, ctypes.c_int] + [_dp] * 4
        L.kgpu_fp64_peak.argtypes = [_dp]
        L.kgpu_eval_powers.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.kgpu_rad_implicit_cells_warm_device.argtypes = [ctypes.c_int, rpp] + [vp] * 13 + [
            ctypes.POINTER(ctypes.c_ulonglong)]
        sop = ctypes.POINTER(SolverOpts)
        L.kgpu_rad_implicit_cells_device_ex.argtypes = [ctypes.c_int, rpp] + [vp] * 11 + [
            ctypes.c_int, sop, vp, vp, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]
        cfp = ctypes.POINTER(Config)
        L.kgpu_u2p_cells_device.argtypes = [ctypes.c_int, cfp, ctypes.c_int] + [vp] * 5 + [ctypes.c_float] * 2 + [
            vp] * 4 + [ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int]
        L.kgpu_u2p_features_device.argtypes = [ctypes.c_int, cfp, ctypes.c_int] + [vp] * 6
        L.kgpu_u2p_targets_device.argtypes = [ctypes.c_int, cfp, ctypes.c_int] + [vp] * 7
        L.kgpu_rad_default_solver_opts.argtypes = [sop]
        L.kgpu_rad_set_solver_opts.argtypes = [sop]
        L.kgpu_rad_get_solver_opts.argtypes = [sop]
        L.kgpu_set_implicit_options.argtypes = [vp, sop]
        L.kgpu_get_implicit_options.argtypes = [vp, sop]
        tup = ctypes.POINTER(Tuning)
        L.kgpu_get_tuning.argtypes = [vp, tup]
        L.kgpu_set_tuning.argtypes = [vp, tup]
        L.kgpu_autotune.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, tup, _dp]
        L.kgpu_tune_select.argtypes = [ctypes.c_int, _dp, ctypes.c_int, ctypes.c_double]
        L.kgpu_rad_features_device.argtypes = [ctypes.c_int, rpp] + [vp] * 6
        L.kgpu_rad_targets_device.argtypes = [ctypes.c_int, rpp] + [vp] * 8
        fp = ctypes.POINTER(ctypes.c_float)
        L.kgpu_mlp_create.argtypes = [ctypes.POINTER(vp), ctypes.c_ulonglong]
        L.kgpu_mlp_destroy.argtypes = [vp]
        L.kgpu_mlp_get.argtypes = [vp, fp]
        L.kgpu_mlp_set.argtypes = [vp, fp]
        L.kgpu_mlp_forward.argtypes = [vp, vp, ctypes.c_int, vp, vp]
        L.kgpu_mlp_gradient.argtypes = [vp, vp, vp, ctypes.c_int, fp, _dp]
        L.kgpu_mlp_train_epoch.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                           ctypes.c_ulonglong, _dp]
        L.kgpu_u2p_cells_static.argtypes = sig["kgpu_u2p_cells"]
        L.kgpu_u2p_cells_full.argtypes = [ctypes.c_int, ctypes.POINTER(Config), rpp, _dp, _dp, _dp, _dp,
                                          ip_, ip_, ip_]
        L.kgpu_addi_u_3.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.kgpu_do_correct.argtypes = [vp]
        L.kgpu_flux_ct.argtypes = [vp]
        for name, args in (("kgpu_fm_radtorus_state", [ctypes.POINTER(TorusParams), rpp, ctypes.c_double,
                                                        ctypes.POINTER(Config)] + [_dp] * 7),
                           ("kgpu_init_fm_radtorus", [vp, ctypes.POINTER(TorusParams), rpp, ctypes.c_double,
                                                      ctypes.c_int]),
                           ("kgpu_init_fm_radtorus_host", [vp, ctypes.POINTER(TorusParams), rpp, ctypes.c_double,
                                                           ctypes.c_int]),
                           ("kgpu_get_implicit_buffers", [vp, ctypes.POINTER(ctypes.c_int)] +
                            [ctypes.POINTER(vp)] * 9),
                           ("kgpu_set_radiation", [vp, rpp, ctypes.c_int]),
                           ("kgpu_set_implicit_solver", [vp, ctypes.c_int, vp]),
                           ("kgpu_set_warm_gate", [vp, ctypes.c_int]),
                           ("kgpu_rk2imex_steps", [vp, ctypes.c_int]),
                           ("kgpu_rk2imex_steps_graph", [vp, ctypes.c_int])):
            getattr(L, name).argtypes = args
            getattr(L, name).restype = ctypes.c_int
        L.kgpu_u2p_cells_static.restype = ctypes.c_int
        L.kgpu_u2p_cells_static_error.restype = ctypes.c_char_p
        L.kgpu_abi_version.restype = ctypes.c_int
        _LIB = L
    return _LIB


def _check(rc, what):
    if rc != 0:
        msg = lib().kgpu_last_error().decode(errors="replace")
        raise KgpuError(f"{what} failed with code {rc}: {msg}")


def _ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def default_config(nx, ny, nz, **kw):
    c = Config()
    _check(lib().kgpu_default_config(ctypes.byref(c), nx, ny, nz), "kgpu_default_config")
    for k, v in kw.items():
        if k == "bc":
            for i in range(3):
                c.bc[i] = int(v[i])
        else:
            setattr(c, k, v)
    return c


class Subdomain:
    """One KORAL tile resident on the current GPU.

    Methods are named after the reference routines they replace and keep
    their argument meaning (finite.c:501-2620, ko.c:290-626).
    """

    def __init__(self, cfg):
        self.cfg = cfg
        self.L = lib()
        h = ctypes.c_void_p()
        _check(self.L.kgpu_create(ctypes.byref(cfg), ctypes.byref(h)), "kgpu_create")
        self.h = h
        ng = cfg.ng
        self.sx = cfg.nx + 2 * ng
        self.sy = cfg.ny + 2 * ng if cfg.ny > 1 else 1
        self.sz = cfg.nz + 2 * ng if cfg.nz > 1 else 1
        self.nv = cfg.nv

    def close(self):
        if getattr(self, "h", None):
            self.L.kgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return (self.sz, self.sy, self.sx, self.nv)

    # set-up
    def set_uniform_grid(self, lo, hi):
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        hi = np.ascontiguousarray(hi, dtype=np.float64)
        _check(self.L.kgpu_set_uniform_grid(self.h, _ptr(lo), _ptr(hi)), "kgpu_set_uniform_grid")

    def upload_grid(self, xbx, xby, xbz):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (xbx, xby, xbz)]
        _check(self.L.kgpu_upload_grid(self.h, *[_ptr(x) for x in a]), "kgpu_upload_grid")

    def set_density_floor(self, centres, xfaces):
        if centres is None:
            _check(self.L.kgpu_set_density_floor(self.h, None, None), "kgpu_set_density_floor")
            return
        c = np.ascontiguousarray(centres, dtype=np.float64)
        f = np.ascontiguousarray(xfaces, dtype=np.float64)
        _check(self.L.kgpu_set_density_floor(self.h, _ptr(c), _ptr(f)), "kgpu_set_density_floor")

    def set_minkowski_metric(self):
        _check(self.L.kgpu_set_minkowski_metric(self.h), "kgpu_set_minkowski_metric")

    def upload_metric(self, g, G, gKr, gbx, gby, gbz, Gbx, Gby, Gbz):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (g, G, gKr, gbx, gby, gbz, Gbx, Gby, Gbz)]
        _check(self.L.kgpu_upload_metric(self.h, *[_ptr(x) for x in a]), "kgpu_upload_metric")

    def calc_scalars(self, spin=0.9, mass=10.0, bhdisk=False, t=0.):
        """calc_scalars of the black-hole disk computed on the device
        (NSCALARS values; the header documents each entry)."""
        sp = ScalarsParams(float(spin), float(mass), int(bool(bhdisk)))
        out = np.zeros(NSCALARS)
        _check(self.L.kgpu_calc_scalars(self.h, ctypes.byref(sp), float(t), _ptr(out)), "kgpu_calc_scalars")
        return out

    def set_polar_correction(self, flags, nc=2):
        """The polar-axis corrections of do_correct (POLAR_CORRECT,
        POLAR_CORRECT_3D, POLAR_SMOOTH bits; nc = NCCORRECTPOLAR)."""
        _check(self.L.kgpu_set_polar_correction(self.h, int(flags), int(nc)), "kgpu_set_polar_correction")

    # time averages (save_avg, fileop.c:10-70)
    def set_avg(self, on=True, mass=10.0):
        """Allocate the averages; with on, the fused steps call save_avg once
        per step (AVGOUTPUT=1).  mass (solar masses) sets the units of the
        averaged temperature when there is no radiation."""
        _check(self.L.kgpu_set_avg(self.h, int(bool(on)), float(mass)), "kgpu_set_avg")

    def save_avg(self, dt):
        _check(self.L.kgpu_save_avg(self.h, float(dt)), "kgpu_save_avg")

    def reset_avg(self):
        _check(self.L.kgpu_reset_avg(self.h), "kgpu_reset_avg")

    def download_avg(self):
        """(pavg [SZ][SY][SX][NV+NAVGVARS], avgtime)"""
        nav = self.L.kgpu_avg_count(self.h)
        if nav < 0:
            _check(nav, "kgpu_avg_count")
        out = np.zeros(self.shape[:3] + (nav,))
        t = ctypes.c_double()
        _check(self.L.kgpu_download_avg(self.h, _ptr(out), ctypes.byref(t)), "kgpu_download_avg")
        return out, t.value

    def download_metric(self):
        """The metric tables in KORAL's layout, in the argument order of
        upload_metric."""
        out = [np.zeros(n) for n in _metric_sizes(self.cfg)]
        _check(self.L.kgpu_download_metric(self.h, *[_ptr(o) for o in out]), "kgpu_download_metric")
        return out

    def init_fm_torus(self, tp=None, on_host=False):
        """Grid, metric, density floor, torus state, boundaries and first dt.
        The metric and the state are computed on the device; on_host=True
        computes them with the host functions and uploads them."""
        tp = tp or torus_params()
        name = "kgpu_init_fm_torus_host" if on_host else "kgpu_init_fm_torus"
        _check(getattr(self.L, name)(self.h, ctypes.byref(tp)), name)

    def init_orszag_tang(self):
        _check(self.L.kgpu_init_orszag_tang(self.h), "kgpu_init_orszag_tang")

    # state transfer
    def upload_state(self, u, p):
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(self.shape)
        p = np.ascontiguousarray(p, dtype=np.float64).reshape(self.shape)
        _check(self.L.kgpu_upload_state(self.h, _ptr(u), _ptr(p)), "kgpu_upload_state")

    def download_state(self):
        u = np.empty(self.shape)
        p = np.empty(self.shape)
        _check(self.L.kgpu_download_state(self.h, _ptr(u), _ptr(p)), "kgpu_download_state")
        return u, p

    def download_flux(self, d):
        nf = [(self.sx + 1) * self.sy * self.sz, self.sx * (self.sy + 1) * self.sz, self.sx * self.sy * (self.sz + 1)][d]
        a = np.empty((nf, self.nv))
        _check(self.L.kgpu_download_flux(self.h, d, _ptr(a)), "kgpu_download_flux")
        return a

    def download_emf(self):
        c = self.cfg
        a = np.empty(((c.nx + 1) * (c.ny + 1) * (c.nz + 1), 3))
        _check(self.L.kgpu_download_emf(self.h, _ptr(a)), "kgpu_download_emf")
        return a

    def download(self, which):
        a = np.empty(self.shape)
        _check(self.L.kgpu_download_array(self.h, which, _ptr(a)), "kgpu_download_array")
        return a

    # KORAL operators
    def op_explicit(self, t, dt):
        _check(self.L.kgpu_op_explicit(self.h, t, dt), "kgpu_op_explicit")

    def op_implicit(self, t, dt):
        _check(self.L.kgpu_op_implicit(self.h, t, dt), "kgpu_op_implicit")

    def calc_u2p(self):
        _check(self.L.kgpu_calc_u2p(self.h), "kgpu_calc_u2p")

    def set_bc(self, t=0.0, ifinit=0):
        _check(self.L.kgpu_set_bc(self.h, t, ifinit), "kgpu_set_bc")

    def save_timesteps(self):
        _check(self.L.kgpu_save_timesteps(self.h), "kgpu_save_timesteps")

    def copyi_u(self, factor, src, dst):
        _check(self.L.kgpu_copyi_u(self.h, factor, src, dst), "kgpu_copyi_u")

    def addi_u(self, f1, a, f2, b, c):
        _check(self.L.kgpu_addi_u(self.h, f1, a, f2, b, c), "kgpu_addi_u")

    # time-step bookkeeping
    def addi_u_3(self, f1, a, f2, b, f3, c, d):
        _check(self.L.kgpu_addi_u_3(self.h, f1, a, f2, b, f3, c, d), "kgpu_addi_u_3")

    def do_correct(self):
        _check(self.L.kgpu_do_correct(self.h), "kgpu_do_correct")

    def flux_ct(self):
        """flux_ct (magn.c:199): stores the rewritten magnetic face fluxes
        of the last op_explicit (kgpu_flux_ct)."""
        _check(self.L.kgpu_flux_ct(self.h), "kgpu_flux_ct")

    def begin_run(self):
        _check(self.L.kgpu_begin_run(self.h), "kgpu_begin_run")

    def begin_step(self):
        dt = ctypes.c_double()
        _check(self.L.kgpu_begin_step(self.h, ctypes.byref(dt)), "kgpu_begin_step")
        return dt.value

    @property
    def tstepdenmax(self):
        v = ctypes.c_double()
        _check(self.L.kgpu_get_tstepdenmax(self.h, ctypes.byref(v)), "kgpu_get_tstepdenmax")
        return v.value

    @tstepdenmax.setter
    def tstepdenmax(self, v):
        _check(self.L.kgpu_set_tstepdenmax(self.h, float(v)), "kgpu_set_tstepdenmax")

    def rk2_steps(self, n=1, graph=False):
        fn = self.L.kgpu_rk2_steps_graph if graph else self.L.kgpu_rk2_steps
        _check(fn(self.h, int(n)), "kgpu_rk2_steps")

    def counters(self):
        a = (ctypes.c_ulonglong * 20)()
        n = self.L.kgpu_get_counters_ex(self.h, a, 20)
        if n < 0:
            _check(n, "kgpu_get_counters_ex")
        return dict(fixups=a[0], entropy=a[1], failed=a[2], negrho=a[3], iters_energy=a[4], iters_entropy=a[5],
                    paused=a[6], to_entropy=a[7], rad_corrected=a[8], radimp_failed=a[9], imp_iters=a[10],
                    imp_passes=a[11], imp_fallbacks=a[12], imp_evals=a[13], imp_inner=a[14], imp_inner_f=a[15],
                    imp_cooperative=a[16], imp_solves=a[17], rad_floors=a[18], face_floors=a[19])

    def set_radiation(self, rp, wavespeed_limiter=False):
        """Radiation in the step (nv = 13): M1 fluxes and speeds, u2p_rad and
        radiation floors, the implicit source operator (kgpu_set_radiation)."""
        self._rp = rp
        _check(self.L.kgpu_set_radiation(self.h, ctypes.byref(rp), int(bool(wavespeed_limiter))),
               "kgpu_set_radiation")

    def set_implicit_solver(self, mode=None, warm=None):
        """Solver of op_implicit (RAD_PLAIN, RAD_BATCHED or RAD_PERSISTENT)
        and the warm-start network (an Mlp, kept alive by this object), or
        None."""
        mode = RAD_BATCHED if mode is None else mode
        self._warm = warm
        _check(self.L.kgpu_set_implicit_solver(self.h, int(mode), warm.h if warm is not None else None),
               "kgpu_set_implicit_solver")

    def write_restart(self, folder, nout1, t, nout2=0, problem=0):
        """res%04d.head/.dat in the reference's format (fprint_restartfile_bin)."""
        _check(self.L.kgpu_write_restart(self.h, os.fsencode(folder), int(nout1), int(nout2), float(t), int(problem)),
               "kgpu_write_restart")

    def read_restart(self, folder, nout1=-1):
        """Reads a restart file (nout1 < 0: reslast); returns (t, next nout1, nout2)."""
        t = ctypes.c_double()
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(self.L.kgpu_read_restart(self.h, os.fsencode(folder), int(nout1), ctypes.byref(t), ctypes.byref(a),
                                        ctypes.byref(b)), "kgpu_read_restart")
        return t.value, a.value, b.value

    def implicit_buffers(self):
        """Device pointers of the last implicit step's buffers: n and a dict of
        pp_in, uu_in, pp_out ([n][13] doubles), g20, G20 ([n][20]), dt ([n]),
        status, attempt, iters ([n] int32)."""
        n = ctypes.c_int()
        ptrs = [ctypes.c_void_p() for _ in range(9)]
        _check(self.L.kgpu_get_implicit_buffers(self.h, ctypes.byref(n), *[ctypes.byref(q) for q in ptrs]),
               "kgpu_get_implicit_buffers")
        names = ("pp_in", "uu_in", "pp_out", "g20", "G20", "dt", "status", "attempt", "iters")
        return n.value, {k: q.value for k, q in zip(names, ptrs)}

    def implicit_pairs(self, rp):
        """Warm-start network inputs and training targets (float device
        tensors [n][16] and [n][5], targets NaN where the solve failed) of the
        cells of the last implicit step."""
        import torch
        n, b = self.implicit_buffers()
        X = torch.empty((n, 16), dtype=torch.float32, device="cuda")
        T = torch.empty((n, MLP_OUT), dtype=torch.float32, device="cuda")
        vp = ctypes.c_void_p
        _check(self.L.kgpu_rad_features_device(n, ctypes.byref(rp), vp(b["pp_in"]), vp(b["g20"]), vp(b["G20"]),
                                               vp(b["dt"]), _vp(X), _stream()), "kgpu_rad_features_device")
        _check(self.L.kgpu_rad_targets_device(n, ctypes.byref(rp), vp(b["pp_in"]), vp(b["pp_out"]), vp(b["g20"]),
                                              vp(b["G20"]), vp(b["status"]), vp(b["attempt"]), _vp(T), _stream()),
               "kgpu_rad_targets_device")
        return X, T

    def implicit_options(self):
        """This context's solver tuning (a SolverOpts)."""
        o = SolverOpts()
        _check(self.L.kgpu_get_implicit_options(self.h, ctypes.byref(o)), "kgpu_get_implicit_options")
        return o

    def set_implicit_options(self, opts=None, **kw):
        """Set this context's solver tuning: a SolverOpts, or fields changed
        by keyword from the current values."""
        o = self.implicit_options() if opts is None else opts
        for k, v in kw.items():
            setattr(o, k, int(v))
        _check(self.L.kgpu_set_implicit_options(self.h, ctypes.byref(o)), "kgpu_set_implicit_options")

    def tuning(self):
        t = Tuning()
        _check(self.L.kgpu_get_tuning(self.h, ctypes.byref(t)), "kgpu_get_tuning")
        return t

    def set_tuning(self, t):
        _check(self.L.kgpu_set_tuning(self.h, ctypes.byref(t)), "kgpu_set_tuning")

    def autotune(self, steps=2, min_gain=0.02, reuse=False):
        """kgpu_autotune: times candidate launch shapes and solver settings
        on this context's state (restored afterwards), applies and returns
        the choice with the time per step before and after (ms)."""
        t = Tuning()
        ms = (ctypes.c_double * 2)()
        _check(self.L.kgpu_autotune(self.h, int(steps), float(min_gain), int(bool(reuse)), ctypes.byref(t), ms),
               "kgpu_autotune")
        return t, (ms[0], ms[1])

    def set_warm_gate(self, iters):
        """Warm-start only cells whose previous solve took a later attempt or
        more than `iters` Newton iterations (-1: every cell)."""
        _check(self.L.kgpu_set_warm_gate(self.h, int(iters)), "kgpu_set_warm_gate")

    def rk2imex_steps(self, n=1, graph=False):
        fn = self.L.kgpu_rk2imex_steps_graph if graph else self.L.kgpu_rk2imex_steps
        _check(fn(self.h, int(n)), "kgpu_rk2imex_steps")

    def set_u2p_pass_iters(self, n):
        _check(self.L.kgpu_set_u2p_pass_iters(self.h, int(n)), "kgpu_set_u2p_pass_iters")

    @property
    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        v = ctypes.c_void_p()
        _check(self.L.kgpu_get_stream(self.h, ctypes.byref(v)), "kgpu_get_stream")
        return v.value or 0

    def profile(self, on=True):
        _check(self.L.kgpu_profile_enable(self.h, int(on)), "kgpu_profile_enable")

    def profile_reset(self):
        _check(self.L.kgpu_profile_reset(self.h), "kgpu_profile_reset")

    def profile_read(self):
        """{kernel name: (total ms, launches)} since the last reset."""
        out = {}
        for k in range(self.L.kgpu_num_kernels()):
            ms = ctypes.c_double()
            n = ctypes.c_longlong()
            nm = ctypes.c_char_p()
            _check(self.L.kgpu_profile_read(self.h, k, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(nm)),
                   "kgpu_profile_read")
            out[nm.value.decode()] = (ms.value, n.value)
        return out

    @property
    def launches(self):
        v = ctypes.c_longlong()
        _check(self.L.kgpu_launch_count(self.h, ctypes.byref(v)), "kgpu_launch_count")
        return v.value

    def reset_counters(self):
        _check(self.L.kgpu_reset_counters(self.h), "kgpu_reset_counters")


def orszag_tang(n=128, graph_ok=True):
    """Relativistic Orszag-Tang vortex on an n x n periodic grid."""
    cfg = default_config(n, n, 1, ng=3, int_order=PPM, fluxmethod=LAXF, gamma=5.0 / 3.0, tsteplim=0.5)
    s = Subdomain(cfg)
    s.set_uniform_grid([0.0, 0.0, -1.0], [2 * np.pi, 2 * np.pi, 1.0])
    s.set_minkowski_metric()
    s.init_orszag_tang()
    s.begin_run()
    return s


def u2p_cells(cfg, uu, pp, g, G):
    """Batched u2p (u2p.c:176) of n independent cells; returns (pp, status, fixup)."""
    uu = np.ascontiguousarray(uu, dtype=np.float64)
    pp = np.ascontiguousarray(pp, dtype=np.float64).copy()
    g = np.ascontiguousarray(g, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    n = uu.shape[0]
    st = np.zeros(n, dtype=np.int32)
    fx = np.zeros(n, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    _check(lib().kgpu_u2p_cells(n, ctypes.byref(cfg), _ptr(uu), _ptr(pp), _ptr(g), _ptr(G),
                                st.ctypes.data_as(ip), fx.ctypes.data_as(ip)), "kgpu_u2p_cells")
    return pp, st, fx


STATIC_MAX_CELLS = 8192   # KGPU_STATIC_MAX_CELLS


def u2p_cells_static(cfg, uu, pp, g, G):
    """u2p_cells through kgpu_u2p_cells_static, which allocates no device
    memory: at most STATIC_MAX_CELLS cells per call, calls share one device
    array and must not overlap on the GPU."""
    uu = np.ascontiguousarray(uu, dtype=np.float64)
    pp = np.ascontiguousarray(pp, dtype=np.float64).copy()
    g = np.ascontiguousarray(g, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    n = uu.shape[0]
    st = np.zeros(n, dtype=np.int32)
    fx = np.zeros(n, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    L = lib()
    rc = L.kgpu_u2p_cells_static(n, ctypes.byref(cfg), _ptr(uu), _ptr(pp), _ptr(g), _ptr(G),
                                 st.ctypes.data_as(ip), fx.ctypes.data_as(ip))
    if rc != 0:
        msg = L.kgpu_u2p_cells_static_error().decode(errors="replace")
        raise KgpuError(f"kgpu_u2p_cells_static failed with code {rc}: {msg}")
    return pp, st, fx


def u2p_cells_full(cfg, uu, pp, g, G, rp=None):
    """The reference's per-cell u2p with all outputs (kgpu_u2p_cells_full):
    returns (pp, status, corrected [n][3], fixups [n][2])."""
    uu, pp, g, G = (np.ascontiguousarray(a, dtype=np.float64) for a in (uu, pp, g, G))
    n = uu.shape[0]
    pp = pp.copy()
    st = np.zeros(n, np.int32)
    co, fx = np.zeros((n, 3), np.int32), np.zeros((n, 2), np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    _check(lib().kgpu_u2p_cells_full(n, ctypes.byref(cfg), ctypes.byref(rp) if rp is not None else None, _ptr(uu),
                                     _ptr(pp), _ptr(g), _ptr(G), st.ctypes.data_as(ip), co.ctypes.data_as(ip),
                                     fx.ctypes.data_as(ip)), "kgpu_u2p_cells_full")
    return pp, st, co, fx


def eval_powers(kind, x, y=0.0):
    """kgpu_eval_powers on the device: kind 0 x^2, 1 x^4, 2 x^-3.5, 3 x^y
    (quarter exponents), 4 log, 5 the device library's pow."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    _check(lib().kgpu_eval_powers(len(x), int(kind), float(y), _ptr(x), _ptr(out)), "kgpu_eval_powers")
    return out


def tune_select(ms, incumbent, min_gain=0.02):
    """The autotuner's selection rule (kgpu_tune_select)."""
    a = np.ascontiguousarray(ms, dtype=np.float64)
    r = lib().kgpu_tune_select(len(a), _ptr(a), int(incumbent), float(min_gain))
    if r < 0:
        _check(r, "kgpu_tune_select")
    return r


def p2u_cells(cfg, pp, g, G):
    """Batched p2u (p2u.c:40) of n independent cells."""
    pp = np.ascontiguousarray(pp, dtype=np.float64)
    g = np.ascontiguousarray(g, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    uu = np.empty_like(pp)
    _check(lib().kgpu_p2u_cells(pp.shape[0], ctypes.byref(cfg), _ptr(pp), _ptr(uu), _ptr(g), _ptr(G)),
           "kgpu_p2u_cells")
    return uu


def torus_params(**kw):
    tp = TorusParams()
    _check(lib().kgpu_default_torus_params(ctypes.byref(tp)), "kgpu_default_torus_params")
    for k, v in kw.items():
        setattr(tp, k, v)
    return tp


def torus_config(nx=192, ny=96, nz=64):
    """Config of the magnetised Kerr torus: MP5 + HLL, MKS2 axisymmetric
    metric, outflow / polar reflection / periodic phi boundaries."""
    return default_config(nx, ny, nz, ng=4, int_order=MP5, fluxmethod=HLL, axisym_metric=1,
                          bc=(BC_OUTFLOW, BC_REFLECT, BC_PERIODIC_COPY), gamma=13.0 / 9.0, tsteplim=0.5,
                          uurhoratiomin=1e-10, uurhoratiomax=1e2, b2rhoratiomax=100.0)


def fm_torus(nx=192, ny=96, nz=64, tp=None, on_host=False):
    """The benchmark torus on the current GPU, initialised by the product's
    own metric and Fishbone-Moncrief set-up (computed on the device unless
    on_host)."""
    s = Subdomain(torus_config(nx, ny, nz))
    s.init_fm_torus(tp, on_host=on_host)
    return s


def _metric_sizes(cfg):
    """Sizes of the nine metric tables (g, G, Christoffels, g and G of the
    x, y, z faces) in KORAL's layout."""
    sx = cfg.nx + 2 * cfg.ng
    sy = cfg.ny + 2 * cfg.ng if cfg.ny > 1 else 1
    sz = cfg.nz + 2 * cfg.ng if cfg.nz > 1 else 1
    sm = 1 if cfg.axisym_metric else sz
    return [sx * sy * sm * 20, sx * sy * sm * 20, sx * sy * sm * 64,
            (sx + 1) * sy * sm * 20, sx * (sy + 1) * sm * 20, sx * sy * (sm + 1) * 20,
            (sx + 1) * sy * sm * 20, sx * (sy + 1) * sm * 20, sx * sy * (sm + 1) * 20]


def mks2_metric_tables(tp, cfg, xb):
    """Host-side MKS2 metric tables (KORAL layout) for faces xb = (xbx, xby, xbz)."""
    out = [np.zeros(n) for n in _metric_sizes(cfg)]
    xb = [np.ascontiguousarray(x, dtype=np.float64) for x in xb]
    _check(lib().kgpu_mks2_metric_tables(tp.spin, tp.r0, tp.h0, cfg.nx, cfg.ny, cfg.nz, cfg.ng, cfg.axisym_metric,
                                         *[_ptr(x) for x in xb], *[_ptr(o) for o in out]), "kgpu_mks2_metric_tables")
    return out


def fm_torus_state(tp, cfg, xb, g, G):
    sx = cfg.nx + 2 * cfg.ng
    sy = cfg.ny + 2 * cfg.ng
    sz = cfg.nz + 2 * cfg.ng
    u = np.zeros((sz, sy, sx, cfg.nv))
    p = np.zeros((sz, sy, sx, cfg.nv))
    xb = [np.ascontiguousarray(x, dtype=np.float64) for x in xb]
    _check(lib().kgpu_fm_torus_state(ctypes.byref(tp), ctypes.byref(cfg), *[_ptr(x) for x in xb],
                                     _ptr(np.ascontiguousarray(g)), _ptr(np.ascontiguousarray(G)), _ptr(u), _ptr(p)),
           "kgpu_fm_torus_state")
    return u, p


def fm_radtorus_state(tp, rp, eradatm, cfg, xb, g, G):
    """The radiative torus state (nv = 13), host arrays in KORAL layout."""
    sx, sy, sz = cfg.nx + 2 * cfg.ng, cfg.ny + 2 * cfg.ng, cfg.nz + 2 * cfg.ng
    u = np.zeros((sz, sy, sx, cfg.nv))
    p = np.zeros((sz, sy, sx, cfg.nv))
    xb = [np.ascontiguousarray(x, dtype=np.float64) for x in xb]
    _check(lib().kgpu_fm_radtorus_state(ctypes.byref(tp), ctypes.byref(rp), float(eradatm), ctypes.byref(cfg),
                                        *[_ptr(x) for x in xb], _ptr(np.ascontiguousarray(g)),
                                        _ptr(np.ascontiguousarray(G)), _ptr(u), _ptr(p)),
           "kgpu_fm_radtorus_state")
    return u, p


RADTORUS_MASS = 1.e16      # black-hole mass (Msun) of the radiative torus: sets the radiation units
RADTORUS_ERADATM = 1.e-6   # atmosphere radiation energy relative to its gas energy


def radtorus_config(nx=256, ny=128, nz=64):
    """The torus configuration with M1 radiation (13 variables)."""
    cfg = torus_config(nx, ny, nz)
    cfg.nv = 13
    return cfg


def radtorus(nx=256, ny=128, nz=64, tp=None, rp=None, eradatm=RADTORUS_ERADATM, wavespeed_limiter=False,
             on_host=False):
    """A Subdomain holding the radiative torus, radiation switched on; metric
    and state computed on the device unless on_host."""
    tp = tp or torus_params()
    rp = rp or rad_params(mass=RADTORUS_MASS, gamma=13.0 / 9.0)
    s = Subdomain(radtorus_config(nx, ny, nz))
    s._rp = rp
    name = "kgpu_init_fm_radtorus_host" if on_host else "kgpu_init_fm_radtorus"
    _check(getattr(lib(), name)(s.h, ctypes.byref(tp), ctypes.byref(rp), float(eradatm),
                                int(bool(wavespeed_limiter))), name)
    return s


# ---------------------------------------------------------------------------
# radiation: per-cell implicit gas-radiation source solve
# ---------------------------------------------------------------------------
RAD_PLAIN, RAD_BATCHED, RAD_PERSISTENT = 0, 1, 2
NVR = 13


def solver_opts(**kw):
    """kgpu_rad_default_solver_opts with fields changed by keyword."""
    o = SolverOpts()
    _check(lib().kgpu_rad_default_solver_opts(ctypes.byref(o)), "kgpu_rad_default_solver_opts")
    for k, v in kw.items():
        setattr(o, k, int(v))
    return o


def rad_params(mass=10.0, gamma=13.0 / 9.0, kramers=6.4e22, kes=0.34):
    """Constants and solver controls (KORAL's defaults) for a black hole of
    `mass` solar masses and a Kramers + electron-scattering opacity law."""
    rp = RadParams()
    _check(lib().kgpu_rad_default_params(ctypes.byref(rp), mass, gamma, kramers, kes), "kgpu_rad_default_params")
    return rp


def _cells(*arrs):
    return [np.ascontiguousarray(a, dtype=np.float64) for a in arrs]


def rad_implicit_cells(rp, uu, pp, g, G, dt, mode=RAD_BATCHED):
    """solve_implicit_lab (rad.c:1225) on n independent cells; returns
    (pp, uu, status, attempt, iters)."""
    uu, pp, g, G, dt = _cells(uu, pp, g, G, dt)
    n = uu.shape[0]
    po, uo = np.zeros_like(pp), np.zeros_like(uu)
    st, at, it = (np.zeros(n, dtype=np.int32) for _ in range(3))
    ip = ctypes.POINTER(ctypes.c_int)
    _check(lib().kgpu_rad_implicit_cells(n, ctypes.byref(rp), _ptr(uu), _ptr(pp), _ptr(g), _ptr(G), _ptr(dt),
                                         _ptr(po), _ptr(uo), st.ctypes.data_as(ip), at.ctypes.data_as(ip),
                                         it.ctypes.data_as(ip), mode), "kgpu_rad_implicit_cells")
    return po, uo, st, at, it


def rad_u2p_cells(rp, uu, pp, g, G):
    """u2p_rad (u2prad.c:485) on n cells; returns (pp, status, corrected)."""
    uu, pp, g, G = _cells(uu, pp, g, G)
    pp = pp.copy()
    n = uu.shape[0]
    st, co = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    _check(lib().kgpu_rad_u2p_cells(n, ctypes.byref(rp), _ptr(uu), _ptr(pp), _ptr(g), _ptr(G),
                                    st.ctypes.data_as(ip), co.ctypes.data_as(ip)), "kgpu_rad_u2p_cells")
    return pp, st, co


def rad_p2u_cells(rp, pp, g, G):
    """p2u (p2u.c:40) of the 13-variable state on n cells."""
    pp, g, G = _cells(pp, g, G)
    uu = np.zeros_like(pp)
    _check(lib().kgpu_rad_p2u_cells(pp.shape[0], ctypes.byref(rp), _ptr(pp), _ptr(uu), _ptr(g), _ptr(G)),
           "kgpu_rad_p2u_cells")
    return uu


def ks_metric(a, r, th):
    """Kerr-Schild metric point in the 20 + 20 layout."""
    g20, G20 = np.zeros(20), np.zeros(20)
    _check(lib().kgpu_ks_metric(a, r, th, _ptr(g20), _ptr(G20)), "kgpu_ks_metric")
    return g20, G20


def rad_cell_draws(n, seed, rp, metric=None, spin=0.9, sigma=None):
    """Random radiating cells around a Kerr black hole: r log-uniform in
    [2, 100] M, theta uniform in [0.1, pi - 0.1]; log-uniform rho in
    [1e-8, 1], gas temperature in [1e4, 1e12] K, E_rad/rho in [1e-10, 1e2]
    and optical depth per cell in [1e-3, 1e5]; gas Lorentz factor
    log-uniform in [1, 20] and radiation flux fraction uniform in [0, 0.99],
    each in an isotropic direction; with sigma = (lo, hi), a magnetic field
    in an isotropic direction with B^i g_ij B^j / rho log-uniform in
    [lo, hi].  Returns (pp, g, G, tau) with the entropy
    slot of pp left for the caller (it goes with the conserved variables).
    `metric(r, th)` gives the metric point (default: the product's
    Kerr-Schild metric)."""
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(2.), np.log(100.), n))
    th = rng.uniform(0.1, np.pi - 0.1, n)
    g20, G20 = np.zeros((n, 20)), np.zeros((n, 20))
    if metric is None:
        _check(lib().kgpu_ks_metric_batch(spin, n, _ptr(r), _ptr(th), _ptr(g20), _ptr(G20)), "kgpu_ks_metric_batch")
    else:
        for k in range(n):
            g20[k], G20[k] = metric(r[k], th[k])
    rho = 10 ** rng.uniform(-8, 0, n)
    T = 10 ** rng.uniform(4, 12, n)
    u = rp.kb * rho * T / rp.mu / rp.mp / (rp.gamma - 1.)
    Erf = 10 ** rng.uniform(-10, 2, n) * rho

    def direction(norm2):
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        v = d / np.sqrt(np.stack([g20[:, 6], g20[:, 12], g20[:, 18]], 1))
        vgv = np.einsum('ni,nij,nj->n', v, g20.reshape(n, 4, 5)[:, 1:4, 1:4], v)
        return v * np.sqrt(norm2 / vgv)[:, None]

    gam = np.exp(rng.uniform(0., np.log(20.), n))
    ug = direction(gam ** 2 - 1.)
    f = rng.uniform(0., 0.99, n)
    vr = np.where(f > 0, (4. - np.sqrt(16. - 12. * f * f)) / (2. * np.maximum(f, 1e-300)), 0.)
    ur = direction(vr * vr / (1. - vr * vr))
    pp = np.zeros((n, NVR))
    pp[:, 0], pp[:, 1], pp[:, 2:5], pp[:, 9], pp[:, 10:13] = rho, u, ug, Erf, ur
    tau = 10 ** rng.uniform(-3, 5, n)
    if sigma is not None:
        sg = 10 ** rng.uniform(np.log10(sigma[0]), np.log10(sigma[1]), n)
        pp[:, 6:9] = direction(sg * rho)
    return pp, g20, G20, tau


def rad_cells(n, seed, rp, spin=0.9, metric=None, sigma=None):
    """rad_cell_draws completed with the product's own p2u: entropy, conserved
    variables, and dt = 0.5 dx with dx = tau / (kappa_abs + kappa_es) (the
    light-crossing CFL step of a cell of that optical depth).  Returns
    (uu, pp, g, G, dt)."""
    pp, g20, G20, tau = rad_cell_draws(n, seed, rp, metric=metric, spin=spin, sigma=sigma)
    gm1 = rp.gamma - 1.
    idx = 1. / gm1
    pp[:, 5] = pp[:, 0] * np.log((gm1 * pp[:, 1]) ** idx / pp[:, 0] ** (idx + 1.))
    uu = rad_p2u_cells(rp, pp, g20, G20)
    T = pp[:, 1] * gm1 / (rp.kb * pp[:, 0] / rp.mu / rp.mp)
    rhocgs = pp[:, 0] / rp.ggg * rp.ccc * rp.ccc / rp.masscm / rp.masscm
    kabs = rp.kramers * rhocgs * T ** -3.5 / rp.ggg * rp.ccc * rp.ccc / rp.masscm * pp[:, 0]
    kes = rp.kes_gu * pp[:, 0]
    dt = 0.5 * tau / (kabs + kes)
    return uu, pp, g20, G20, dt


# ---------------------------------------------------------------------------
# learned warm start (device tensors from torch: plumbing only)
# ---------------------------------------------------------------------------
def _vp(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p()


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Mlp:
    """The warm-start network (kgpu_mlp_*): 16 -> 128 -> 128 -> 5, SiLU,
    BF16 tensor-core kernels with FP32 accumulation."""

    def __init__(self, seed=1):
        self.L = lib()
        self.h = ctypes.c_void_p()
        _check(self.L.kgpu_mlp_create(ctypes.byref(self.h), seed), "kgpu_mlp_create")
        self.size = self.L.kgpu_mlp_blob_size()

    def close(self):
        if self.h:
            self.L.kgpu_mlp_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get(self):
        b = np.zeros(self.size, dtype=np.float32)
        _check(self.L.kgpu_mlp_get(self.h, b.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), "kgpu_mlp_get")
        return b

    def set(self, blob):
        b = np.ascontiguousarray(blob, dtype=np.float32)
        assert b.size == self.size
        _check(self.L.kgpu_mlp_set(self.h, b.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), "kgpu_mlp_set")

    def forward(self, X):
        import torch
        Y = torch.empty((X.shape[0], 8), dtype=torch.float32, device=X.device)
        _check(self.L.kgpu_mlp_forward(self.h, _vp(X), X.shape[0], _vp(Y), _stream()), "kgpu_mlp_forward")
        return Y

    def gradient(self, X, T):
        g = np.zeros(self.size - 16, dtype=np.float32)
        loss = ctypes.c_double()
        _check(self.L.kgpu_mlp_gradient(self.h, _vp(X), _vp(T), X.shape[0],
                                        g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(loss)),
               "kgpu_mlp_gradient")
        return g, loss.value

    def train_epoch(self, X, T, batch=8192, lr=1e-3, seed=0):
        loss = ctypes.c_double()
        _check(self.L.kgpu_mlp_train_epoch(self.h, _vp(X), _vp(T), X.shape[0], batch, lr, seed,
                                           ctypes.byref(loss)), "kgpu_mlp_train_epoch")
        return loss.value


def rad_features_device(rp, pp, g, G, dt):
    import torch
    X = torch.empty((pp.shape[0], 16), dtype=torch.float32, device=pp.device)
    _check(lib().kgpu_rad_features_device(pp.shape[0], ctypes.byref(rp), _vp(pp), _vp(g), _vp(G), _vp(dt), _vp(X),
                                          _stream()), "kgpu_rad_features_device")
    return X


MLP_OUT = 7   # network outputs: five for the initial iterate, two attempt scores


def rad_targets_device(rp, pp, pp1, g, G, status, attempt):
    """Training targets [n][7] of solved cells (kgpu_rad_targets_device)."""
    import torch
    T = torch.empty((pp.shape[0], MLP_OUT), dtype=torch.float32, device=pp.device)
    _check(lib().kgpu_rad_targets_device(pp.shape[0], ctypes.byref(rp), _vp(pp), _vp(pp1), _vp(g), _vp(G),
                                         _vp(status), _vp(attempt), _vp(T), _stream()), "kgpu_rad_targets_device")
    return T


U2P_WGATE, U2P_SGATE = 0.005, 0.5   # default gates of the u2p warm start (measured best on held-out cells)


def u2p_cells_device(cfg, uu, pp, g, G, ypred=None, wgate=U2P_WGATE, sgate=U2P_SGATE):
    """The MHD inversion of n cells on device tensors (kgpu_u2p_cells_device):
    uu, pp [n][nv] (nine MHD variables first), g, G [n][20]; pp is the guess.
    With ypred (the network's output on u2p_features_device), the learned
    warm start: the predicted W where |ln(W/W_guess)| >= wgate, the entropy
    equation alone where the score passes sgate.  Returns (pp, status,
    fixup, iters, stats) with stats = [Newton iterations, fallbacks,
    W-function evaluations]."""
    import torch
    n, nv = uu.shape
    dev = uu.device
    po = pp.clone()
    st, fx, it = (torch.empty(n, dtype=torch.int32, device=dev) for _ in range(3))
    stats = (ctypes.c_ulonglong * 3)()
    _check(lib().kgpu_u2p_cells_device(n, ctypes.byref(cfg), nv, _vp(uu), _vp(po), _vp(g), _vp(G),
                                       _vp(ypred) if ypred is not None else None, float(wgate), float(sgate),
                                       _vp(st), _vp(fx), _vp(it),
                                       _stream(), stats, 3), "kgpu_u2p_cells_device")
    return po, st, fx, it, list(stats)


def u2p_features_device(cfg, uu, pp, g, G):
    """Network inputs [n][16] of the u2p warm start (kgpu_u2p_features_device)."""
    import torch
    n, nv = uu.shape
    X = torch.empty((n, 16), dtype=torch.float32, device=uu.device)
    _check(lib().kgpu_u2p_features_device(n, ctypes.byref(cfg), nv, _vp(uu), _vp(pp), _vp(g), _vp(G), _vp(X),
                                          _stream()), "kgpu_u2p_features_device")
    return X


def u2p_targets_device(cfg, pp, pp1, g, G, status):
    """Training targets [n][7] of the u2p warm start (kgpu_u2p_targets_device)."""
    import torch
    n, nv = pp.shape
    T = torch.empty((n, MLP_OUT), dtype=torch.float32, device=pp.device)
    _check(lib().kgpu_u2p_targets_device(n, ctypes.byref(cfg), nv, _vp(pp), _vp(pp1), _vp(g), _vp(G), _vp(status),
                                         _vp(T), _stream()), "kgpu_u2p_targets_device")
    return T


def u2p_config(gamma, u2pconv=1e-10, rhofloor=1e-50):
    """A Config carrying the inversion's parameters (GAMMA, U2PCONV, the
    density floor) for the per-cell u2p entry points."""
    cfg = default_config(1, 1, 1, ng=3, gamma=gamma)
    cfg.u2pconv = u2pconv
    cfg.rhofloor = rhofloor
    return cfg


def rad_solve_device(rp, uu, pp, g, G, dt, mode=RAD_BATCHED, ypred=None, work=None, opts=None, nstats=3):
    """Implicit solve on device tensors (kgpu_rad_implicit_cells_device_ex);
    with ypred, the learned warm start; opts a SolverOpts or None for the
    process-wide values.  Returns (pp, uu, status, attempt, iters, stats)
    with nstats counters (Newton iterations, launches with work, warm-start
    fallbacks, evaluations, nested Newton steps, nested W evaluations,
    evaluations handed to a warp)."""
    import torch
    n = uu.shape[0]
    dev = uu.device
    po = torch.empty_like(pp)
    uo = torch.empty_like(uu)
    st, at, it = (torch.empty(n, dtype=torch.int32, device=dev) for _ in range(3))
    L = lib()
    if work is None and mode != RAD_PLAIN:
        work = torch.empty(int(L.kgpu_rad_work_bytes(n)), dtype=torch.uint8, device=dev)
    stats = (ctypes.c_ulonglong * nstats)()
    _check(L.kgpu_rad_implicit_cells_device_ex(n, ctypes.byref(rp), _vp(uu), _vp(pp), _vp(g), _vp(G), _vp(dt),
                                               _vp(ypred) if ypred is not None else None, _vp(po), _vp(uo),
                                               _vp(st), _vp(at), _vp(it), mode,
                                               ctypes.byref(opts) if opts is not None else None,
                                               _vp(work) if work is not None else None, _stream(), stats, nstats),
           "kgpu_rad_implicit_cells_device_ex")
    return po, uo, st, at, it, list(stats)

