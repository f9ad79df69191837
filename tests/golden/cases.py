"""Seeded synthetic job inputs in the reference's own formats.

Each case is a job dictionary with the reference's params.json keys plus the arrays
the reference reads from its input files:

  fxyz    (3, NZ, NY) float32  -- the Fault_geometry file (x, y, z of the fault surface,
                                  coord.cu:71-151; the grid is that surface extruded in x)
  stress  (15, NZ, NY) float32 -- the Fault_init_stress file planes
                                  Tx,Ty,Tz,dTx,dTy,dTz,mu_s,mu_d,Dc,C0,a,b,L,Vw,State
                                  (init.cu:904-1005)
  layers  (n, 4) float32       -- a Media1D table depth,rho,vp,vs (media.cu:63-138)
  wave0   (9, nx, nz, ny) f64  -- optional initial wavefield (volume-only checks)

The fault-surface and stress formulas restate the reference's job scripts
(jobs/tpv3_free_dh100m/conf_fault_grid.m:1-49, conf_fault_stress.m:42-152,
jobs/tpv10_new/conf_fault_stress.m) in numpy; the public benchmark data they are
compared with in the reference (SCEC TPV FEM traces) are not used anywhere.
"""
import json
import os

import numpy as np


def flat_geometry(NY, NZ, DH):
    """Planar vertical fault x=0 (conf_fault_grid.m:15-22, 0-based indices)."""
    j = np.arange(NY)[None, :]
    k = np.arange(NZ)[:, None]
    x = np.zeros((NZ, NY))
    y = (j - NY / 2) * DH + 0 * k
    z = (k + 1 - NZ) * DH + 0 * j
    return np.stack([x, y, z]).astype(np.float32)


def curved_geometry(NY, NZ, DH, dip_deg=60.0, hill_amp=500.0, hill_width=5e3, nhills=2, seed=0):
    """Dipping planar fault meshed by a curvilinear grid with Gaussian-hill topography
    on the free surface: the surface height varies along strike (the reference grid is
    the fault surface extruded along x, coord.cu:299-311) and is tapered linearly to a
    flat bottom.  The dip offsets x by depth / tan(dip) (the TPV10 geometry, coord.cu:257-260)."""
    rng = np.random.default_rng(seed)
    j = np.arange(NY)[None, :].astype(np.float64)
    k = np.arange(NZ)[:, None].astype(np.float64)
    y = (j - NY / 2) * DH + 0 * k
    top = np.zeros_like(j)
    for _ in range(nhills):
        yc = rng.uniform(-0.3, 0.3) * NY * DH
        amp = hill_amp * rng.uniform(0.5, 1.0)
        top = top + amp * np.exp(-((j - NY / 2) * DH - yc) ** 2 / hill_width ** 2)
    depth_flat = (NZ - 1 - k) * DH  # depth below z=0 on a flat surface
    zbot = -(NZ - 1) * DH
    frac = k / (NZ - 1)
    z = zbot + frac * (0 - zbot) + frac * top  # bottom flat, top follows the hills
    depth = np.maximum(-z, 0.0)
    x = depth / np.tan(np.deg2rad(dip_deg)) - depth_flat.mean() / np.tan(np.deg2rad(dip_deg))
    return np.stack([x, y + 0 * k, z + 0 * j]).astype(np.float32)


def rough_geometry(NY, NZ, DH, ratio=1e-3, lmin=1e3, hurst=1.0, seed=0):
    """Vertical fault with seeded self-similar roughness x(y, z): a Gaussian random field
    with isotropic power spectrum P(k) ~ k^-(2 hurst + 2) (hurst = 1: self-similar), cut
    at the minimum wavelength lmin by a 4-pole low-pass, scaled so that its rms height is
    ratio x the strike length (the amplitude-to-wavelength ratio of a self-similar surface,
    after jobs/tpv3_free_dh100m/func_selfsimilar2d.m)."""
    fx = flat_geometry(NY, NZ, DH).astype(np.float64)
    rng = np.random.default_rng(seed)
    ky = np.fft.fftfreq(NY, d=DH)[None, :]
    kz = np.fft.fftfreq(NZ, d=DH)[:, None]
    k = np.sqrt(ky ** 2 + kz ** 2)
    amp = np.zeros_like(k)
    nz = k > 0
    amp[nz] = k[nz] ** (-(hurst + 1.0)) / np.sqrt(1.0 + (k[nz] * lmin) ** 8)
    h = np.real(np.fft.ifft2(np.fft.fft2(rng.standard_normal((NZ, NY))) * amp))
    h *= ratio * NY * DH / h.std()
    fx[0] = h
    return fx.astype(np.float32)


def surface_normal(fxyz, DH):
    """Unit normal of the fault surface x(y,z) from central differences (the base
    vector the reference's job scripts project the stress tensor on)."""
    x, y, z = [a.astype(np.float64) for a in fxyz]
    ty = np.stack([np.gradient(x, axis=1), np.gradient(y, axis=1), np.gradient(z, axis=1)])
    tz = np.stack([np.gradient(x, axis=0), np.gradient(y, axis=0), np.gradient(z, axis=0)])
    n = np.cross(ty, tz, axis=0)
    n /= np.linalg.norm(n, axis=0, keepdims=True)
    n *= np.sign(n[0:1])  # +x side
    return n


def sw_stress(fxyz, Fault_grid, tn=-120e6, ts=-70e6, patch=None, patch_ts=-81.6e6, mu_s=0.677, mu_d=0.525,
              Dc=0.4, C0=0.0, outside_mu_s=1000.0, outside_C0=1000e6, normal=None):
    """Slip-weakening initial traction and friction planes (conf_fault_stress.m:42-126)."""
    _, NZ, NY = fxyz.shape
    y, z = fxyz[1].astype(np.float64), fxyz[2].astype(np.float64)
    n = np.zeros((3, NZ, NY)); n[0] = 1.0
    if normal is not None:
        n = normal
    sxy = np.full((NZ, NY), ts)
    if patch is not None:
        yc, zc, hw = patch
        inside = (np.abs(y - yc) < hw) & (np.abs(z - zc) < hw)
        sxy[inside] = patch_ts
    # traction = sigma . n with sigma = [[tn, sxy, 0], [sxy, 0, 0], [0, 0, 0]]
    Tx = tn * n[0] + sxy * n[1]
    Ty = sxy * n[0]
    Tz = np.zeros_like(Tx)
    out = np.zeros((15, NZ, NY))
    out[0], out[1], out[2] = Tx, Ty, Tz
    j1, j2, k1, k2 = Fault_grid
    ms = np.full((NZ, NY), outside_mu_s)
    c0 = np.full((NZ, NY), outside_C0)
    ms[k1 - 1:k2, j1 - 1:j2] = mu_s
    c0[k1 - 1:k2, j1 - 1:j2] = C0
    out[6], out[7], out[8], out[9] = ms, mu_d, Dc, c0
    return out.astype(np.float32)


def depth_stress(fxyz, Fault_grid, grad=7378.0, ratio=0.55, normal=None, mu_s=0.76, mu_d=0.448, Dc=0.5, C0=0.2e6,
                 patch=None):
    """Depth-dependent stress (TPV10 style, jobs/tpv10_new/conf_fault_stress.m): normal
    stress grad*depth, shear = ratio*normal along the dip direction, nucleation patch at
    (mu_s+0.0057)*normal."""
    _, NZ, NY = fxyz.shape
    z = fxyz[2].astype(np.float64)
    depth = np.maximum(-z, 0.5 * 100.0)
    n = normal if normal is not None else np.stack([np.ones_like(z), 0 * z, 0 * z])
    # dip direction: the in-plane tangent orthogonal to strike (y)
    ey = np.stack([0 * z, np.ones_like(z), 0 * z])
    d = np.cross(n, ey, axis=0)
    d /= np.linalg.norm(d, axis=0, keepdims=True)
    d *= -np.sign(d[2:3] + 1e-30)  # pointing down-dip
    sn = -grad * depth
    tau = ratio * np.abs(sn)
    if patch is not None:
        yc, zc, hw = patch
        y = fxyz[1].astype(np.float64)
        inside = (np.abs(y - yc) < hw) & (np.abs(z - zc) < hw)
        tau = np.where(inside, (mu_s + 0.0057) * np.abs(sn) + 0.2e6, tau)
    T = sn * n + tau * d
    out = np.zeros((15, NZ, NY))
    out[0:3] = T
    j1, j2, k1, k2 = Fault_grid
    ms = np.full((NZ, NY), 1000.0)
    c0 = np.full((NZ, NY), 1000e6)
    ms[k1 - 1:k2, j1 - 1:j2] = mu_s
    c0[k1 - 1:k2, j1 - 1:j2] = C0
    out[6], out[7], out[8], out[9] = ms, mu_d, Dc, c0
    return out.astype(np.float32)


def rs_fields(stress, fxyz, a_range=(0.01, 0.02), b=0.014, L=0.4, Vw=0.1, V0=1e-6, Vini=1e-16, seed=0,
              normal=None, patch=None, patch_dtau=25e6):
    """Rate-and-state planes (conf_fault_stress.m:127-152): a log-uniform per node,
    steady-state initial state psi = a ln(2 V0/Vini sinh(|tau|/(|sigma_n| a)))."""
    rng = np.random.default_rng(seed)
    _, NZ, NY = fxyz.shape
    lo, hi = np.log(a_range[0]), np.log(a_range[1])
    a = np.exp(rng.uniform(lo, hi, size=(NZ, NY)))
    out = stress.astype(np.float64).copy()
    n = normal if normal is not None else np.stack([np.ones((NZ, NY)), np.zeros((NZ, NY)), np.zeros((NZ, NY))])
    T = out[0:3]
    tn = (T * n).sum(0)
    ts = np.linalg.norm(T - tn * n, axis=0)
    psi = a * np.log(2.0 * V0 / Vini * np.sinh(ts / np.abs(tn) / a))
    out[10], out[11], out[12], out[13], out[14] = a, b, L, Vw, psi
    if patch is not None:
        yc, zc, hw = patch
        y, z = fxyz[1].astype(np.float64), fxyz[2].astype(np.float64)
        r = np.sqrt((y - yc) ** 2 + (z - zc) ** 2)
        with np.errstate(over="ignore", divide="ignore"):
            F = np.where(r < hw, np.exp(np.minimum(r ** 2 / (r ** 2 - hw ** 2 + 1e-30), 0.0)), 0.0)
        sdir = (T - tn * n) / np.maximum(ts, 1.0)
        out[3:6] = patch_dtau * F * sdir
    return out.astype(np.float32)


def smooth_wave(NX, NY, NZ, seed=0, amp=1e5):
    """Seeded smooth initial wavefield with zero ghost layers (9, nx, nz, ny)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = NX + 6, NY + 6, NZ + 6
    W = np.zeros((9, nx, nz, ny))
    i = np.arange(nx)[:, None, None]
    k = np.arange(nz)[None, :, None]
    j = np.arange(ny)[None, None, :]
    for f in range(9):
        ci, cj, ck = rng.uniform(0.3, 0.7, 3) * np.array([nx, ny, nz])
        w = rng.uniform(2.0, 4.0)
        scale = amp if f >= 3 else amp * 1e-6
        W[f] = scale * np.exp(-((i - ci) ** 2 + (j - cj) ** 2 + (k - ck) ** 2) / (2 * w * w))
    W[:, :3] = 0; W[:, -3:] = 0
    W[:, :, :3] = 0; W[:, :, -3:] = 0
    W[:, :, :, :3] = 0; W[:, :, :, -3:] = 0
    return W


def get_case(name):
    """Return (params, fxyz, stress, layers, wave0, meta) for a named case."""
    if name == "vol_small":
        p = dict(NX=20, NY=22, NZ=18, DH=100.0, DT=0.004, TMAX=0.05, PML_N=5, PML_velocity=6000.0,
                 INPORT_GRID_TYPE=0)
        return p, None, None, None, smooth_wave(20, 22, 18, seed=1), dict(steps=12, every=4, volume=True)
    if name == "vol_curved":
        p = dict(NX=20, NY=24, NZ=18, DH=100.0, DT=0.004, TMAX=0.05, PML_N=5, PML_velocity=6000.0,
                 INPORT_GRID_TYPE=1, bi_vp2=5000.0, bi_vs2=2900.0, bi_rho2=2500.0)
        fx = curved_geometry(24, 18, 100.0, hill_amp=300.0, hill_width=600.0, seed=3)
        return p, fx, None, None, smooth_wave(20, 24, 18, seed=2), dict(steps=12, every=4, volume=True)
    if name in ("sw_flat", "sw_flat_nr"):
        NX, NY, NZ, DH = 24, 76, 40, 100.0
        fg = [21, 56, 21, 40]
        p = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.008, TMAX=0.4, PML_N=6, PML_velocity=6000.0,
                 INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=0, Fault_grid=fg,
                 mu_s=0.677, mu_d=0.525, Dc=0.4, C0=0.0, NormalRefine=1 if name == "sw_flat" else 0)
        fx = flat_geometry(NY, NZ, DH)
        st = sw_stress(fx, fg, patch=(0.0, -500.0, 450.0), patch_ts=-95e6, Dc=0.05, mu_d=0.525)
        return p, fx, st, None, None, dict(steps=60, every=20, volume=False)
    if name == "sw_cerjan":
        # slip weakening with the Cerjan sponge on top of the PML (reference -DuseCerjan)
        NX, NY, NZ, DH = 24, 76, 40, 100.0
        fg = [21, 56, 21, 40]
        p = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.008, TMAX=0.4, PML_N=6, PML_velocity=6000.0,
                 INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=0, Fault_grid=fg,
                 mu_s=0.677, mu_d=0.525, Dc=0.4, C0=0.0, useCerjan=1, DAMP_N=8)
        fx = flat_geometry(NY, NZ, DH)
        st = sw_stress(fx, fg, patch=(0.0, -500.0, 450.0), patch_ts=-95e6, Dc=0.05, mu_d=0.525)
        return p, fx, st, None, None, dict(steps=60, every=20, volume=False)
    if name == "sw_curved":
        NX, NY, NZ, DH = 24, 76, 40, 100.0
        fg = [21, 56, 21, 40]
        p = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.006, TMAX=0.3, PML_N=6, PML_velocity=6000.0,
                 INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=0, Fault_grid=fg,
                 mu_s=0.76, mu_d=0.448, Dc=0.05, C0=0.2e6)
        fx = curved_geometry(NY, NZ, DH, hill_amp=200.0, hill_width=800.0, seed=5)
        n = surface_normal(fx, DH)
        st = depth_stress(fx, fg, normal=n, Dc=0.05, patch=(0.0, -500.0, 450.0))
        return p, fx, st, None, None, dict(steps=50, every=25, volume=False)
    if name == "rs_flat":
        NX, NY, NZ, DH = 24, 76, 40, 100.0
        fg = [21, 56, 21, 40]
        p = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.008, TMAX=0.32, PML_N=6, PML_velocity=6000.0,
                 INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=2, Fault_grid=fg,
                 RS_V0=1e-6, RS_f0=0.6, RS_fw=0.2, RS_Vini=1e-16, RS_L=0.4, smooth_load_T=0.1)
        fx = flat_geometry(NY, NZ, DH)
        st = sw_stress(fx, fg, tn=-120e6, ts=-40e6)
        st = rs_fields(st, fx, seed=7, L=0.02, patch=(0.0, -500.0, 600.0), patch_dtau=45e6)
        return p, fx, st, None, None, dict(steps=40, every=20, volume=False)
    if name == "rs_aging":
        # rs_flat with the aging law (Friction_type 1, rk4.cu:899-901)
        p, fx, st, layers, w0, meta = get_case("rs_flat")
        p["Friction_type"] = 1
        return p, fx, st, layers, w0, meta
    if name == "tp_flat":
        # rs_flat with thermal pressurisation: 64 points per column, so that the diffusion
        # sub-cycles (sub-step 10/63^2 s < DT), hydraulic diffusivity log-uniform per node
        p, fx, st, layers, w0, meta = get_case("rs_flat")
        p.update(Friction_type=3, TP_n=64)
        rng = np.random.default_rng(11)
        hy = np.exp(rng.uniform(np.log(2e-5), np.log(4e-4), size=st.shape[1:])).astype(np.float32)
        return p, fx, np.concatenate([st, hy[None]]), layers, w0, meta
    if name == "rs_rough":
        return rs_rough_case(76, 24, 40, seed=31, L=0.02, steps=60)
    if name == "rs_curved":
        # the rough fault of rs_rough loaded over 0.05 s, so that it ruptures within its 40
        # steps: the wavefield then stands far above the FP32 rounding of the traction
        # rebuilt from the curved fault's varying normals (~10 Pa of 120 MPa)
        p, fx, st, layers, w0, meta = rs_rough_case(76, 24, 40, seed=31, L=0.02, steps=40)
        p["smooth_load_T"] = 0.05
        return p, fx, st, layers, w0, dict(meta, every=20)
    if name == "media_cj":
        return media_case()
    raise KeyError(name)


def media_case(NX=56, NY=100, NZ=60, DH=50.0, steps=80):
    """The large-domain configuration in miniature: a 1-D layered medium from a Media1D
    table (vs 2000 to 3600 m/s and rho 2400 to 2800 kg/m^3 over depth, vp = sqrt(3) vs),
    a 20-node PML with a 20-node Cerjan sponge beside it, a non-planar fault (smooth
    along-strike and down-dip bumps of the fault surface x(y, z)) meshed by the curvilinear
    grid, DH = 50 m, and a slip-weakening rupture (TPV10-style depth-dependent stress and
    friction) nucleated at 700 m depth.  Layer depths
    lie between node depths so that the layer each node takes does not hinge on rounding.
    The reference's FP64 build cannot read a Media1D table (media.cu:84 scans "%g" into
    double), so this case has an FP32 reference fixture only."""
    fg = [31, NY - 30, 31, NZ]
    p = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.004, TMAX=steps * 0.004 + 0.002, PML_N=20, PML_velocity=6236.0,
             INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=0, Fault_grid=fg, mu_s=0.76,
             mu_d=0.448, Dc=0.01, C0=0.2e6, useCerjan=1, DAMP_N=20)
    fx = flat_geometry(NY, NZ, DH).astype(np.float64)
    j = np.arange(NY)[None, :]
    k = np.arange(NZ)[:, None]
    fx[0] = 60.0 * np.sin(2 * np.pi * 1.3 * j / NY + 0.4) + 30.0 * np.cos(2 * np.pi * 0.6 * k / NZ)
    fx = fx.astype(np.float32)
    n = surface_normal(fx, DH)
    st = depth_stress(fx, fg, normal=n, Dc=0.01, patch=(0.0, -700.0, 400.0))
    depth = np.array([0.0, 325.0, 625.0, 925.0, 1225.0, 1525.0, 2025.0])
    vs = np.linspace(2000.0, 3600.0, depth.size)
    rho = np.linspace(2400.0, 2800.0, depth.size)
    layers = np.stack([depth, rho, np.sqrt(3.0) * vs, vs], 1).astype(np.float32)
    return p, fx, st, layers, None, dict(steps=steps, every=steps // 2, volume=False, variants=("sp",),
                                         jblock=(36, 72))


def write_media1d(fn, layers):
    """A Media1D text file as init_media1d reads it (media.cu:63-90): a comment line, the
    layer count, a column header, then one 'depth rho vp vs' row per layer."""
    with open(fn, "w") as f:
        f.write("# 1-D layered medium\n")
        f.write(f"{len(layers)}\n")
        f.write("depth rho vp vs\n")
        for row in np.asarray(layers, np.float32):
            f.write(" ".join(f"{float(v):.9g}" for v in row) + "\n")


def rs_rough_case(NY, NX, NZ, seed=0, DH=100.0, steps=40, L=0.4):
    """Rate-and-state slip law on a seeded self-similar rough fault (the learned-guess
    configuration): a log-uniform in [0.01, 0.02] per node, b = 0.014, L = 0.4 m,
    V0 = 1e-6 m/s, f0 = 0.6, fw = 0.2, Vw = 0.1 m/s, Vini = 1e-16 m/s; normal stress
    120 MPa, shear 40 MPa, a 45 MPa nucleation patch of 3 km radius at 7.5 km depth (600 m
    at 500 m depth on small grids) loaded over smooth_load_T.  The small test grid uses a
    shorter L so that it slips within its few steps."""
    fg = [1, NY, 1, NZ]
    p = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=0.008, TMAX=steps * 0.008 + 0.004, PML_N=min(12, NX // 4),
             PML_velocity=6000.0, INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Friction_type=2, Fault_grid=fg,
             RS_V0=1e-6, RS_f0=0.6, RS_fw=0.2, RS_Vini=1e-16, RS_L=0.4, smooth_load_T=0.5, NormalRefine=0)
    fx = rough_geometry(NY, NZ, DH, seed=seed)
    n = surface_normal(fx, DH)
    st = sw_stress(fx, fg, tn=-120e6, ts=-40e6)
    # the patch lies inside the non-united area (30-node borders below and along strike)
    depth, radius = (7.5e3, 3.0e3) if NZ * DH >= 1.2e4 else (500.0, 600.0)
    st = rs_fields(st, fx, seed=seed + 1, L=L, normal=n, patch=(0.0, -depth, radius), patch_dtau=45e6)
    return p, fx, st, None, None, dict(steps=steps, every=steps // 2, volume=False)


def ensemble_case(i, seed=2025, size=(100, 300), DH=100.0, DT=0.008, steps=1000):
    """Scenario i of the batched-ensemble configuration: grid size per axis drawn from
    size, stress drop uniform in 2-8 MPa and Dc (slip weakening) or L (rate and state)
    uniform in 0.2-0.8 m from the seed; even scenarios slip weakening, odd ones rate and
    state (slip law); planar fault, homogeneous medium, PML 12, free surface."""
    rng = np.random.default_rng([seed, i])
    NX, NY, NZ = (int(v) for v in rng.integers(size[0], size[1] + 1, 3))
    drop = rng.uniform(2e6, 8e6)
    dc = rng.uniform(0.2, 0.8)
    fg = [31, NY - 30, 31, NZ]
    depth = min(7.5e3, 0.4 * (NZ - 31) * DH)
    radius = min(1.5e3, 0.15 * (NY - 60) * DH)
    p = dict(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=DT, TMAX=steps * DT + DT / 2, PML_N=12, PML_velocity=6000.0,
             INPORT_GRID_TYPE=1, INPORT_STRESS_TYPE=1, Fault_grid=fg, NormalRefine=0)
    fx = flat_geometry(NY, NZ, DH)
    if i % 2 == 0:
        p.update(Friction_type=0, mu_s=0.677, mu_d=0.525, Dc=dc, C0=0.0)
        tau = 0.525 * 120e6 + drop
        st = sw_stress(fx, fg, tn=-120e6, ts=-tau, patch=(0.0, -depth, radius), patch_ts=-82.5e6, Dc=dc, mu_d=0.525)
    else:
        p.update(Friction_type=2, RS_V0=1e-6, RS_f0=0.6, RS_fw=0.2, RS_Vini=1e-16, RS_L=dc, smooth_load_T=0.5)
        st = sw_stress(fx, fg, tn=-120e6, ts=-(35e6 + drop))
        st = rs_fields(st, fx, seed=seed + i, L=dc, patch=(0.0, -depth, radius), patch_dtau=45e6)
    return p, fx, st


CASES = ["vol_small", "vol_curved", "sw_flat", "sw_flat_nr", "sw_curved", "rs_flat", "sw_cerjan", "tp_flat", "rs_aging",
         "rs_curved", "media_cj"]


def write_inputs(name, outdir):
    """Write params.json, Fault_geometry / Fault_init_stress NetCDF-classic files, the
    Media1D table and the optional initial wavefield for the reference harness."""
    p, fx, st, layers, w0, meta = get_case(name)
    return write_job(outdir, p, fx, st, layers, w0), meta


def write_job(outdir, p, fx=None, st=None, layers=None, w0=None):
    """Write a job (parameters and input arrays) in the reference's file formats; returns
    the params.json dictionary."""
    from scipy.io import netcdf_file

    os.makedirs(outdir, exist_ok=True)
    job = dict(p)
    job["OUT"] = outdir
    job["PX"] = job["PY"] = job["PZ"] = 1
    if fx is not None:
        fn = os.path.join(outdir, "fault_coord.nc")
        with netcdf_file(fn, "w") as f:
            f.createDimension("nz", fx.shape[1])
            f.createDimension("ny", fx.shape[2])
            for c, nm in enumerate("xyz"):
                v = f.createVariable(nm, "f4", ("nz", "ny"))
                v[:] = fx[c]
        job["Fault_geometry"] = fn
    if st is not None:
        fn = os.path.join(outdir, "init_stress.nc")
        names = ["Tx", "Ty", "Tz", "dTx", "dTy", "dTz", "mu_s", "mu_d", "Dc", "C0", "a", "b", "L", "Vw", "State",
                 "TP_hy"][:st.shape[0]]
        with netcdf_file(fn, "w") as f:
            f.createDimension("nz", st.shape[1])
            f.createDimension("ny", st.shape[2])
            for c, nm in enumerate(names):
                v = f.createVariable(nm, "f4", ("nz", "ny"))
                v[:] = st[c]
        job["Fault_init_stress"] = fn
    if layers is not None:
        fn = os.path.join(outdir, "media1d.txt")
        write_media1d(fn, layers)
        job["Media1D"] = fn
    with open(os.path.join(outdir, "params.json"), "w") as f:
        json.dump(job, f, indent=1)
    if w0 is not None:
        w0.astype(np.float64).tofile(os.path.join(outdir, "wave0.f64"))
    return job
