"""ctypes wrapper of the CPU oracle (liboracle.so) -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this
module.  It restates the reference's algorithm on the CPU; the product never calls it.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

# Reference parameter defaults (set_params.cu:60-103 and :263-267, which resets the
# PML defaults before reading the job file) plus the reference Makefile's default
# compile-time switches (Makefile:57-161) as runtime flags.
DEFAULTS = dict(
    NX=100, NY=90, NZ=80, TMAX=1.0, DT=0.01, DH=100.0,
    INPORT_GRID_TYPE=0, INPORT_STRESS_TYPE=0, Friction_type=0,
    PML_N=20, PML_velocity=3000.0, PML_bmax=3.0, PML_fc=1.0, DAMP_N=20,
    mu_s=0.677, mu_d=0.525, mu_0=0.0, Dc=0.4, C0=0.0,
    RS_f0=0.0, RS_V0=0.0, RS_Vini=0.0, RS_fw=0.0, RS_L=0.0,
    smooth_load_T=0.0, viscosity=0.0,
    Fault_grid=[0, 0, 0, 0], Asp_grid=[0, 0, 0, 0],
    bi_vp1=6000.0, bi_vs1=3464.0, bi_rho1=2670.0,
    bi_vp2=6000.0, bi_vs2=3464.0, bi_rho2=2670.0,
    FreeSurface=1, usePML=1, useCerjan=0, NormalRefine=1, TP_n=1,
)


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("NX", ctypes.c_int), ("NY", ctypes.c_int), ("NZ", ctypes.c_int), ("NT", ctypes.c_int),
        ("TMAX", ctypes.c_double), ("DT", ctypes.c_double), ("DH", ctypes.c_double),
        ("INPORT_GRID_TYPE", ctypes.c_int), ("INPORT_STRESS_TYPE", ctypes.c_int), ("Friction_type", ctypes.c_int),
        ("PML_N", ctypes.c_int), ("PML_velocity", ctypes.c_double), ("PML_bmax", ctypes.c_double),
        ("PML_fc", ctypes.c_double), ("DAMP_N", ctypes.c_int),
        ("mu_s", ctypes.c_double), ("mu_d", ctypes.c_double), ("mu_0", ctypes.c_double),
        ("Dc", ctypes.c_double), ("C0", ctypes.c_double),
        ("f0", ctypes.c_double), ("V0", ctypes.c_double), ("Vini", ctypes.c_double),
        ("fw", ctypes.c_double), ("L", ctypes.c_double),
        ("smooth_load_T", ctypes.c_double), ("viscosity", ctypes.c_double),
        ("Fault_grid", ctypes.c_int * 4), ("Asp_grid", ctypes.c_int * 4),
        ("bi_vp1", ctypes.c_double), ("bi_vs1", ctypes.c_double), ("bi_rho1", ctypes.c_double),
        ("bi_vp2", ctypes.c_double), ("bi_vs2", ctypes.c_double), ("bi_rho2", ctypes.c_double),
        ("free_surface", ctypes.c_int), ("use_pml", ctypes.c_int), ("use_cerjan", ctypes.c_int),
        ("normal_refine", ctypes.c_int), ("TP_n", ctypes.c_int),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle library not built: run `make -C oracle liboracle.so`")
        _LIB = ctypes.CDLL(path)
        _LIB.orc_create.restype = ctypes.c_void_p
        _LIB.orc_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_int, ctypes.c_void_p]
        _LIB.orc_destroy.argtypes = [ctypes.c_void_p]
        _LIB.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _LIB.orc_step_volume.argtypes = [ctypes.c_void_p, ctypes.c_int]
        _LIB.orc_stage_part.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _LIB.orc_get.restype = ctypes.c_long
        _LIB.orc_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
        _LIB.orc_set.restype = ctypes.c_long
        _LIB.orc_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
        _LIB.orc_newton_iters.restype = ctypes.c_long
        _LIB.orc_newton_iters.argtypes = [ctypes.c_void_p]
        _LIB.orc_threads.restype = ctypes.c_int
    return _LIB


def resolve(params):
    """Apply the reference defaults to a job dictionary (reference JSON keys)."""
    p = dict(DEFAULTS)
    for k, v in params.items():
        if k == "rho1":  # the reference stores "rho1" into bi_rho1 (set_params.cu:247-248)
            p["bi_rho1"] = v
        else:
            p[k] = v
    return p


def to_struct(params):
    p = resolve(params)
    s = OrcParams()
    for name in ("NX", "NY", "NZ", "INPORT_GRID_TYPE", "INPORT_STRESS_TYPE", "Friction_type", "PML_N", "DAMP_N",
                 "TP_n"):
        setattr(s, name, int(p[name]))
    for name in ("TMAX", "DT", "DH", "PML_velocity", "PML_bmax", "PML_fc", "mu_s", "mu_d", "mu_0", "Dc", "C0",
                 "smooth_load_T", "viscosity", "bi_vp1", "bi_vs1", "bi_rho1", "bi_vp2", "bi_vs2", "bi_rho2"):
        setattr(s, name, float(p[name]))
    s.f0, s.V0, s.Vini, s.fw, s.L = (float(p[k]) for k in ("RS_f0", "RS_V0", "RS_Vini", "RS_fw", "RS_L"))
    s.NT = int(float(np.float32(p["TMAX"])) / float(np.float32(p["DT"])))
    for i in range(4):
        s.Fault_grid[i] = int(p["Fault_grid"][i])
        s.Asp_grid[i] = int(p["Asp_grid"][i])
    s.free_surface, s.use_pml = int(p["FreeSurface"]), int(p["usePML"])
    s.use_cerjan, s.normal_refine = int(p["useCerjan"]), int(p["NormalRefine"])
    return s


class Oracle:
    """One simulation held by the CPU oracle.

    fxyz:   (3, NZ, NY) float32 fault-surface coordinates (the Fault_geometry file), or None
    stress: (15, NZ, NY) float32 planes Tx,Ty,Tz,dTx,dTy,dTz,mu_s,mu_d,Dc,C0,a,b,L,Vw,State, or None;
            a 16th plane TP_hy (hydraulic diffusivity, m^2/s) for thermal pressurisation
    layers: (n, 4) float32 rows depth,rho,vp,vs of a 1-D medium (Media1D file), or None
    """

    def __init__(self, params, fxyz=None, stress=None, layers=None, double=True):
        self.params = resolve(params)
        self._s = to_struct(params)
        L = lib()
        self._keep = []

        def ptr(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32)
            self._keep.append(a)
            return a.ctypes.data

        nl = 0 if layers is None else int(np.asarray(layers).shape[0])
        self.h = L.orc_create(ctypes.byref(self._s), 1 if double else 0, ptr(fxyz), ptr(stress), nl, ptr(layers))
        p = self.params
        self.nx, self.ny, self.nz = p["NX"] + 6, p["NY"] + 6, p["NZ"] + 6
        self.nj, self.nk = p["NY"], p["NZ"]
        if stress is not None and np.asarray(stress).shape[0] > 15:
            self.set("TP_hy", np.asarray(stress)[15])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def step(self, it):
        lib().orc_step(self.h, it)

    def stage_part(self, it, irk, part):
        """Part 0 (fault trial), 1 (volume derivatives and PML) or 2 (fault band, RK,
        sponge) of stage irk of step it."""
        lib().orc_stage_part(self.h, it, irk, part)

    def step_volume(self, it):
        lib().orc_step_volume(self.h, it)

    def get(self, name):
        n = lib().orc_get(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        lib().orc_get(self.h, name.encode(), out.ctypes.data)
        return out

    def set(self, name, values):
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        n = lib().orc_set(self.h, name.encode(), v.ctypes.data)
        if n != v.size:
            raise ValueError(f"size mismatch for {name}")

    def wave(self):
        return self.get("W").reshape(9, self.nx, self.nz, self.ny)

    def newton_iters(self):
        return lib().orc_newton_iters(self.h)


def threads():
    return lib().orc_threads()
