"""Named workloads of the pbpic B200 step and their derived parameters.

Units follow the reference (pic2d.f90:15-43, 969-1006): lengths in d_i, time
in 1/Omega_ci, velocities in v_A with c = cva v_A, momenta u = gamma v / c.
For a plasma with frequency ratio wpe/wce and mass ratio mi/me,
c / v_A = (wpe/wce) sqrt(mi/me). The time step is set by a Courant number
C = c dt sqrt(1/dx^2 + 1/dy^2).
"""
import math

from . import _lib as L


def dt_for_cfl(cva, dx, dy, cfl=0.5):
    return cfl / (cva * math.sqrt(1.0 / dx ** 2 + 1.0 / dy ** 2))


def harris_thermal(mime, cva, ti_te):
    """Electron and ion thermal speeds (units of c) of a Harris sheet in
    pressure balance n0 (Ti + Te) = B0^2 / (2 mu0)."""
    te = 1.0 / (2.0 * (1.0 + ti_te))  # Te / (m_i v_A^2)
    vthe = math.sqrt(mime * te) / cva
    vthi = vthe * math.sqrt(ti_te / mime)
    return vthe, vthi


def harris_drifts(lam, cva, ti_te):
    """Drift speeds (units of c) carrying the sheet current: Bx = B0 tanh(y/lambda)
    needs J_z = -(1/lambda) sech^2 in units of n0 e v_A, split as U_i/T_i = -U_e/T_e."""
    du = -1.0 / (lam * cva)  # U_i - U_e
    return du * ti_te / (1.0 + ti_te), -du / (1.0 + ti_te)


def harris_in0(mx, my, dx, dy, ppc, lam, nb):
    """1 / (macro-particles per cell at the sheet peak density n0)."""
    npairs = ppc * mx * my
    lx, ly = mx * dx, my * dy
    cells_equiv = lx * (2.0 * lam + nb * ly) / (dx * dy)
    return cells_equiv / npairs


def uniform_c1(seed=0, mx=128, my=128, ppc=32):
    """Uniform periodic electron-proton plasma: 128x128 cells, dx = dy = 0.05 d_e,
    CFL 0.5, 32 particles per cell per species, mi/me = 25, Ti = Te, electron
    thermal speed 0.1 c, uniform Bz with wpe/wce = 2."""
    mime, cva = 25.0, 2.0 * math.sqrt(25.0)
    dx = dy = 0.05 / math.sqrt(mime)  # 0.05 d_e in d_i
    cfg = dict(mx=mx, my=my, dx=dx, dy=dy, dt=dt_for_cfl(cva, dx, dy), cva=cva, mime=mime,
               in0=1.0 / ppc, ybc=L.BC_PERIODIC)
    vthe = 0.1
    ld = dict(kind=L.LOAD_UNIFORM, ppc=ppc, vthe=vthe, vthi=vthe / math.sqrt(mime), b0z=1.0, seed=seed)
    return cfg, ld


def harris(mx, my, ppc, seed, mime=25.0, wpe_wce=2.0, lam=0.5, nb=0.2, ti_te=5.0, psi0=0.1,
           bguide=0.0, dx=0.1, cfl=0.5):
    cva = wpe_wce * math.sqrt(mime)
    dy = dx
    vthe, vthi = harris_thermal(mime, cva, ti_te)
    udi, ude = harris_drifts(lam, cva, ti_te)
    cfg = dict(mx=mx, my=my, dx=dx, dy=dy, dt=dt_for_cfl(cva, dx, dy, cfl), cva=cva, mime=mime,
               in0=harris_in0(mx, my, dx, dy, ppc, lam, nb), ybc=L.BC_CONDUCTING)
    ld = dict(kind=L.LOAD_HARRIS, ppc=ppc, vthe=vthe, vthi=vthi, vdrift_e=ude, vdrift_i=udi,
              lambda_=lam, nb=nb, psi0=psi0, bguide=bguide, seed=seed)
    return cfg, ld


def double_harris(mx=256, my=256, ppc=64, seed=5, dx=0.04, mime=25.0, cva=15.0, vthec=0.092, lam=0.5,
                  ti_te=5.0, ti_te_bg=1.0, tbg_tcs=0.1, nb=0.2, bguide=0.0, dt=None):
    """The reference's own run (module parameters, pic2d.f90:12-43; initparticles
    and initfields, pic2d.f90:357-648): two current sheets normal to x at Lx/4
    and 3Lx/4, half-thickness lam = 0.5 d_i, on a background nb = 0.2 n0, periodic
    in x and y; 256x256 cells of 0.04 d_i, 64 particle pairs per cell, mi/me = 25,
    c/v_A = 15, dt = 0.045/mime. Sheet electrons have thermal speed vthec c, sheet
    ions Ti/Te = 5; the background is tbg_tcs times as hot, Ti/Te = 1; the sheets
    drift at v_A (ions +z, electrons -z in the first sheet, the reverse in the
    second). in0 = 1/(n0 dx dy) for the sheet peak density n0 (the formula the
    reference keeps beside its hand-set value, pic2d.f90:31-33)."""
    dy = dx
    lx = mx * dx
    vthe_bg = vthec * math.sqrt(tbg_tcs)
    vd = 1.0 / cva
    cfg = dict(mx=mx, my=my, dx=dx, dy=dy, dt=0.045 / mime if dt is None else dt, cva=cva, mime=mime,
               in0=(4.0 * lam + nb * lx) / (ppc * lx), ybc=L.BC_PERIODIC)
    ld = dict(kind=L.LOAD_DOUBLE_HARRIS, ppc=ppc, vthe=vthec, vthi=vthec * math.sqrt(ti_te / mime),
              vthe_bg=vthe_bg, vthi_bg=vthe_bg * math.sqrt(ti_te_bg / mime), vdrift_e=-vd, vdrift_i=vd,
              lambda_=lam, nb=nb, bguide=bguide, seed=seed)
    return cfg, ld


def harris_c2(seed=1, mx=1024, my=512, ppc=100):
    """GEM Harris sheet, 1024x512 cells of 0.1 d_i, 100 particles per cell per
    species (~105M), lambda = 0.5 d_i, nb = 0.2 n0, Ti/Te = 5, wpe/wce = 2,
    psi0 = 0.1 B0 d_i, conducting walls in y, periodic in x."""
    return harris(mx, my, ppc, seed)


def harris_c4(seed=3):
    """The differentiable-form Harris sheet: 256x128 cells, 64 per cell per species."""
    return harris(256, 128, 64, seed)


def harris_c5(seed=4):
    """Large Harris sheet: 4096x2048 cells, 100 per cell per species (~1.68B),
    mi/me = 100, nb = 0.1 n0, guide field 0.2 B0."""
    return harris(4096, 2048, 100, seed, mime=100.0, nb=0.1, bguide=0.2, dx=0.05)


def harris_mid(seed=1):
    """The Harris sheet of harris_c2 on a quarter of the cells (512x256, ~26M
    particles): the profiling case, still far larger than L2."""
    return harris(512, 256, 100, seed)


ENSEMBLE_GRIDS = ((64, 64), (128, 64), (128, 128), (256, 128), (256, 256))


def electron_scale(mx, my, ppc, mime=25.0, wpe_wce=2.0, dx_de=0.05, cfl=0.5):
    """Periodic, unmagnetised electron-scale box: cells of dx_de electron
    inertial lengths, the time step at Courant number cfl."""
    cva = wpe_wce * math.sqrt(mime)
    dx = dx_de / math.sqrt(mime)  # in d_i
    return dict(mx=mx, my=my, dx=dx, dy=dx, dt=dt_for_cfl(cva, dx, dx, cfl), cva=cva, mime=mime,
                in0=1.0 / ppc, ybc=L.BC_PERIODIC)


def two_stream(mx, my, ppc, seed, vdrift=0.2, vthe=0.01):
    """Electron two-stream: beams at +-vdrift c along x, electron thermal
    speed vthe c, immobile neutralising ions."""
    cfg = electron_scale(mx, my, ppc)
    ld = dict(kind=L.LOAD_TWO_STREAM, ppc=ppc, vthe=vthe, vthi=0.0, vdrift_e=vdrift, immobile_ions=1, seed=seed)
    return cfg, ld


def weibel(mx, my, ppc, seed, anisotropy=8.0, vthe=0.1, mime=25.0):
    """Weibel: electrons with T_perp / T_par = anisotropy (perpendicular
    thermal speed vthe c), ions at the parallel electron temperature."""
    cfg = electron_scale(mx, my, ppc, mime=mime)
    vpar = vthe / math.sqrt(anisotropy)
    ld = dict(kind=L.LOAD_WEIBEL, ppc=ppc, vthe=vthe, vthi=vpar / math.sqrt(mime), anisotropy=anisotropy,
              seed=seed)
    return cfg, ld


def ensemble_c3(seed=2, n=64, grids=ENSEMBLE_GRIDS, ppc_range=(16, 128)):
    """The batched ensemble: n instances, grids drawn from `grids`, 16 to 128
    particles per cell per species; even instances two-stream (beams at
    +-0.2 c, thermal 0.01 c), odd ones Weibel (T_perp/T_par = 8, thermal
    0.1 c), drift and anisotropy jittered by +-20 % per instance."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        mx, my = grids[int(rng.integers(len(grids)))]
        ppc = int(rng.integers(ppc_range[0], ppc_range[1] + 1))
        jitter = 1.0 + 0.2 * float(rng.uniform(-1.0, 1.0))
        inst_seed = 1000 * seed + i
        if i % 2 == 0:
            out.append(two_stream(mx, my, ppc, inst_seed, vdrift=0.2 * jitter))
        else:
            out.append(weibel(mx, my, ppc, inst_seed, anisotropy=8.0 * jitter))
    return out


def ensemble_particles(domains):
    return sum(ld["ppc"] * c["mx"] * c["my"] * (1 if ld.get("immobile_ions") else 2) for c, ld in domains)


WORKLOADS = {
    "uniform_128x128_ppc32": uniform_c1,
    "harris_1024x512_ppc100": harris_c2,
    "harris_512x256_ppc100": harris_mid,
    "harris_256x128_ppc64": harris_c4,
    "harris_4096x2048_ppc100": harris_c5,
    "double_harris_256x256_ppc64": double_harris,
}
