"""Seeded synthetic jet set-ups with the shapes of the benchmark configurations.

Host-side numpy initial conditions (the reference has no published datasets;
these follow its own init_block, solvers/srhd3d_mpi_muscl.py:128-160, plus the
magnetised-jet parameters of the RMHD configurations).

    rmhd_jet(n, ng)      RMHD 2 thermo passives (Te, Ti), Gamma = 4/3, ambient
                         rho=1, p=0.01, uniform Bx with sigma=0.01, 1 % seeded
                         velocity noise; the jet (rho=0.1, vx=0.995, W=10.01)
                         enters through the left-x nozzle with a toroidal field.
    srhd_jet(n, ng)      SRHD, ambient rho=1(1 + 1 % noise), p=0.01, at rest;
                         srhd_jet_config gives its nozzle and scheme.
"""
import math

import numpy as np

GAMMA_RMHD = 4.0 / 3.0


def _h(rho, p, gamma):
    return 1.0 + gamma / (gamma - 1.0) * p / rho


def rmhd_jet_config(n, ng=3, vjet=0.995, sigma_amb=0.01, sigma_jet=0.5, radius=0.1,
                    boundaries="reference"):
    """(core params, nozzle cfg, source cfg) of the magnetised jet.

    boundaries="reference": the reference driver's set-up (periodic y/z, fixed
    ambient state on the x = 0 face outside the nozzle, the nozzle's
    "toroidal" field By = B0 s with Bx = 0).  boundaries="baseline": the
    magnetised configurations as specified (outflow on every face but the
    nozzle, a toroidal B_phi = b0 r/R in the jet on the uniform ambient Bx),
    with the library's extensions (astro_outflow_yz, nozzle b_init 3 and
    ambient_bc 1); the nozzle cfg's YZ_BOUNDARY names the y/z fill."""
    W = 1.0 / math.sqrt(1.0 - vjet * vjet)
    rho_j, p_j = 0.1, 0.01
    # comoving b^2 = B^2 / W^2 for a field perpendicular to v
    b0 = W * math.sqrt(sigma_jet * rho_j * _h(rho_j, p_j, GAMMA_RMHD))
    core = dict(GAMMA=GAMMA_RMHD, P_MAX=2.0, V_MAX=0.9999, GLM_CH=1.0, GLM_CP=0.1,
                RECON="weno", LIMITER="mc", RIEMANN="hlld", RK_ORDER=3, CFL=0.35,
                N_PASSIVE=2, PASSIVE_OFFSET=9, RESISTIVE_ENABLED=True, RESISTIVITY=1e-4)
    nozzle = dict(NG=ng, JET_RADIUS=radius, SHEAR_THICK=0.0, NOZZLE_PROFILE="top_hat",
                  GAMMA_JET=W, ETA_RHO=0.1, P_EQ=p_j, RHO_AMB=1.0, VX_AMB=0.0, VY_AMB=0.0,
                  VZ_AMB=0.0, NOZZLE_PERTURB="none", TURB_VAMP=0.0, TURB_PAMP=0.0,
                  PHYSICS="rmhd", B_INIT="toroidal", B0=b0, N_TRACERS=0,
                  TWO_TEMPERATURE=True, THERMO_OFFSET=9, TE_NOZZLE=p_j / rho_j,
                  TI_NOZZLE=p_j / rho_j)
    if boundaries == "baseline":
        nozzle.update(B_INIT="toroidal_phi", NOZZLE_AMBIENT="outflow", YZ_BOUNDARY="outflow",
                      B_AMB_X=math.sqrt(sigma_amb * 1.0 * _h(1.0, 0.01, GAMMA_RMHD)))
    elif boundaries != "reference":
        raise ValueError(boundaries)
    sources = dict(COOLING_ENABLED=True, COOLING_LAMBDA=0.01, HEATING_RATE=0.0, NG=ng,
                   P_MAX=2.0, TWO_TEMPERATURE=True, TEI_TAU=0.1, THERMO_OFFSET=9,
                   N_TRACERS=0)
    return core, nozzle, sources


def rmhd_jet(n, ng=3, seed=2024, sigma_amb=0.01, x_cells=None):
    """Ambient magnetised medium, (11, nx+2ng, n+2ng, n+2ng) float64.  x_cells
    crops the x extent (a slab of the same state, for bounded CPU samples)."""
    rng = np.random.default_rng(seed)
    N = n + 2 * ng
    Nx = (x_cells if x_cells is not None else n) + 2 * ng
    pr = np.zeros((11, Nx, N, N))
    pr[0] = 1.0
    pr[4] = 0.01
    pr[5] = math.sqrt(sigma_amb * 1.0 * _h(1.0, 0.01, GAMMA_RMHD))
    for v in (1, 2, 3):
        pr[v] = 0.01 * (2.0 * rng.random((Nx, N, N)) - 1.0)
    pr[9] = 0.01
    pr[10] = 0.01
    return pr


def srhd_jet_config(n, ng=2, vjet=0.99, recon="muscl", limiter="minmod", riemann="hlle",
                    rk_order=2, cfl=0.4, radius=0.1, boundaries="reference"):
    """(core params, nozzle cfg) of the SRHD jet: Gamma = 5/3, ambient rho = 1
    (1 % noise), p = 0.01 at rest, nozzle rho = 0.1, p = 0.01, vx = vjet on the
    x = 0 face.  The defaults are the 64^3 MUSCL-minmod/HLLE/SSPRK2 set-up;
    vjet=0.995, recon="ppm", riemann="hllc", rk_order=3 the 128^3 one.
    boundaries as in rmhd_jet_config ("baseline": outflow on every face but the
    nozzle)."""
    W = 1.0 / math.sqrt(1.0 - vjet * vjet)
    core = dict(GAMMA=5.0 / 3.0, P_MAX=2.0, V_MAX=0.9999, RECON=recon, LIMITER=limiter,
                RIEMANN=riemann, RK_ORDER=rk_order, CFL=cfl, N_PASSIVE=0, PASSIVE_OFFSET=5)
    nozzle = dict(NG=ng, JET_RADIUS=radius, SHEAR_THICK=0.0, NOZZLE_PROFILE="top_hat",
                  GAMMA_JET=W, ETA_RHO=0.1, P_EQ=0.01, RHO_AMB=1.0, VX_AMB=0.0, VY_AMB=0.0,
                  VZ_AMB=0.0, NOZZLE_PERTURB="none", TURB_VAMP=0.0, TURB_PAMP=0.0,
                  PHYSICS="hydro", B_INIT="none", B0=0.0, N_TRACERS=0,
                  TWO_TEMPERATURE=False)
    if boundaries == "baseline":
        nozzle.update(NOZZLE_AMBIENT="outflow", YZ_BOUNDARY="outflow")
    elif boundaries != "reference":
        raise ValueError(boundaries)
    return core, nozzle


def srhd_jet(n, ng=2, seed=2024):
    rng = np.random.default_rng(seed)
    N = n + 2 * ng
    pr = np.zeros((5, N, N, N))
    pr[0] = 1.0 * (1.0 + 0.01 * (2.0 * rng.random((N, N, N)) - 1.0))
    pr[4] = 0.01
    return pr
