"""Generate the golden parity fixtures from the reference gPLUTO serial build.

Run in a container that has the reference tree (``GP_REFERENCE_ROOT``, by
default ``../reference`` beside the repository):

    python tests/golden/make_golden.py [name ...]

For each case this builds the reference binary (oracle/ref/build_ref.py,
sources compiled in place), writes a seeded initial condition made by
gpluto_dev_b200/ics.py, runs N steps with FTZ/DAZ off, and stores the
initial primitive state, the face fields and the reference's final
Vc/Uc/Vs plus its dt history as ``<name>.npz`` next to this script.
The output/restart cases (``IO_CASES``, stored under ``io/``) also run the
reference with .dbl output every few steps and keep its data.0000.dbl,
data.0001.dbl, dbl.out and restart.out, then restart the reference from
output #1 and store the state it reaches.
The fixtures are small so that they can be committed; the GPU box never
needs the reference tree.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))

from gpluto_dev_b200 import ics  # noqa: E402
import build_ref as br  # noqa: E402

# name: (generator, kwargs, RefConfig kwargs, nsteps)
CASES = {
    "mhd2d_mc_hlld_ucthlld": (ics.mhd2d_turbulence, dict(n=(32, 32), seed=3),
                              dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                   ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4), 20),
    "mhd2d_mc_hlld_ucthlld_long": (ics.mhd2d_turbulence, dict(n=(40, 40), seed=11),
                                   dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                        ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4), 100),
    "mhd2d_vl_hll_ucthll": (ics.mhd2d_turbulence, dict(n=(32, 24), seed=5),
                            dict(physics="MHD", ndim=2, limiter="VANLEER_LIM", solver="hll",
                                 ct_emf="UCT_HLL", cfl=0.4, first_dt=1e-4), 20),
    "mhd2d_mc_hlld_ucthll": (ics.mhd2d_turbulence, dict(n=(24, 32), seed=6),
                             dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                  ct_emf="UCT_HLL", cfl=0.4, first_dt=1e-4), 20),
    "mhd3d_mc_hlld_ucthlld": (ics.mhd3d_turbulence, dict(n=(12, 10, 8), seed=7),
                              dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                   ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4), 10),
    "mhd3d_blast_mc_hlld": (ics.mhd3d_blast, dict(n=(16, 16, 16), seed=2, radius=0.2),
                            dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                 ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4), 12),
    "rmhd3d_mc_hlld_ucthll": (ics.rmhd3d_turbulence, dict(n=(10, 12, 8), seed=12),
                              dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                   ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4), 8),
    "rmhd2d_mc_hlld_ucthll": (ics.rmhd3d_turbulence, dict(n=(24, 20, 2), seed=13),
                              dict(physics="RMHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                   ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4), 16),
    "rmhd3d_vl_hll_ucthll": (ics.rmhd3d_turbulence, dict(n=(8, 10, 12), seed=14, lorentz_max=5.0),
                             dict(physics="RMHD", ndim=3, limiter="VANLEER_LIM", solver="hll",
                                  ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4), 8),
    "hd2d_mc_hllc": (ics.hd_turbulence, dict(n=(32, 32), seed=8),
                     dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc",
                          cfl=0.4, first_dt=1e-4), 20),
    "hd3d_vl_hll": (ics.hd_turbulence, dict(n=(12, 12, 10), seed=9),
                    dict(physics="HD", ndim=3, limiter="VANLEER_LIM", solver="hll",
                         cfl=0.4, first_dt=1e-4), 10),
    # piecewise parabolic reconstruction (RECONSTRUCTION PARABOLIC)
    "mhd2d_ppm_hlld_ucthlld": (ics.mhd2d_turbulence, dict(n=(32, 32), seed=21),
                               dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                    ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                    reconstruction="PARABOLIC"), 20),
    "mhd3d_ppm_hlld_ucthlld": (ics.mhd3d_turbulence, dict(n=(12, 10, 8), seed=22),
                               dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                    ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                    reconstruction="PARABOLIC"), 10),
    "hd2d_ppm_hllc": (ics.hd_turbulence, dict(n=(32, 24), seed=23),
                      dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc",
                           cfl=0.4, first_dt=1e-4, reconstruction="PARABOLIC"), 20),
    # outflow boundaries (HD): x only, all sides with PPM, all sides with VL/HLL
    "hd2d_mc_hllc_outflowx": (ics.hd_turbulence, dict(n=(33, 24), seed=41),
                              dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc",
                                   cfl=0.4, first_dt=1e-4,
                                   bc=("outflow", "periodic", "periodic")), 20),
    "hd3d_ppm_hllc_outflow": (ics.hd_turbulence, dict(n=(12, 10, 9), seed=42),
                              dict(physics="HD", ndim=3, limiter="MC_LIM", solver="hllc",
                                   cfl=0.4, first_dt=1e-4, reconstruction="PARABOLIC",
                                   bc=("outflow", "outflow", "outflow")), 10),
    "hd2d_vl_hll_outflow": (ics.hd_turbulence, dict(n=(24, 32), seed=43),
                            dict(physics="HD", ndim=2, limiter="VANLEER_LIM", solver="hll",
                                 cfl=0.4, first_dt=1e-4,
                                 bc=("outflow", "outflow", "periodic")), 20),
    # outflow boundaries with constrained transport (MHD, RMHD)
    "mhd2d_mc_hlld_ucthlld_outflowx": (ics.mhd2d_turbulence, dict(n=(32, 24), seed=61),
                                       dict(physics="MHD", ndim=2, limiter="MC_LIM",
                                            solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
                                            first_dt=1e-4,
                                            bc=("outflow", "periodic", "periodic")), 20),
    "mhd3d_mc_hlld_ucthlld_outflow": (ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=62),
                                      dict(physics="MHD", ndim=3, limiter="MC_LIM",
                                           solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
                                           first_dt=1e-4,
                                           bc=("outflow", "outflow", "outflow")), 10),
    "mhd2d_ppm_hlld_ucthlld_outflow": (ics.mhd2d_turbulence, dict(n=(24, 28), seed=63),
                                       dict(physics="MHD", ndim=2, limiter="MC_LIM",
                                            solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
                                            first_dt=1e-4, reconstruction="PARABOLIC",
                                            bc=("outflow", "outflow", "periodic")), 16),
    "rmhd3d_mc_hlld_ucthll_outflowz": (ics.rmhd3d_turbulence,
                                       dict(n=(8, 10, 12), seed=64, lorentz_max=3.0),
                                       dict(physics="RMHD", ndim=3, limiter="MC_LIM",
                                            solver="hlld", ct_emf="UCT_HLL", cfl=0.3,
                                            first_dt=1e-4,
                                            bc=("periodic", "periodic", "outflow")), 8),
    "rmhd3d_ppm_hlld_ucthll": (ics.rmhd3d_turbulence,
                               dict(n=(8, 10, 12), seed=24, lorentz_max=3.0),
                               dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                    ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4,
                                    reconstruction="PARABOLIC"), 8),
    # reflective and equatorially symmetric sides (ReflectiveBoundary)
    "mhd2d_mc_hlld_ucthlld_reflectx": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=71),
                                       dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                            ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                            bc=("reflective", "periodic", "periodic")), 12),
    "mhd2d_mc_hlld_ucthlld_reflectx_outflowy": (
        ics.mhd2d_turbulence, dict(n=(24, 20), seed=77),
        dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
             first_dt=1e-4, bc=("reflective", "outflow", "periodic")), 12),
    "mhd2d_vl_hll_ucthll_eqtsymy": (ics.mhd2d_turbulence, dict(n=(20, 24), seed=73),
                                    dict(physics="MHD", ndim=2, limiter="VANLEER_LIM", solver="hll",
                                         ct_emf="UCT_HLL", cfl=0.4, first_dt=1e-4,
                                         bc=("periodic", "eqtsymmetric", "periodic")), 12),
    "mhd3d_blast_mc_hlld_reflect": (ics.mhd3d_blast, dict(n=(14, 12, 10), seed=72, radius=0.25),
                                    dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                         ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                         bc=("reflective", "reflective", "reflective")), 8),
    "hd2d_mc_hllc_reflect": (ics.hd_turbulence, dict(n=(22, 18), seed=74),
                             dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc", cfl=0.4,
                                  first_dt=1e-4, bc=("reflective", "reflective", "periodic")), 12),
    "hd3d_ppm_hllc_reflectz": (ics.hd_turbulence, dict(n=(12, 10, 9), seed=75),
                               dict(physics="HD", ndim=3, limiter="MC_LIM", solver="hllc", cfl=0.4,
                                    first_dt=1e-4, reconstruction="PARABOLIC",
                                    bc=("periodic", "periodic", "reflective")), 8),
    "rmhd3d_mc_hlld_ucthll_reflectx": (ics.rmhd3d_turbulence, dict(n=(10, 8, 8), seed=76,
                                                                   lorentz_max=3.0),
                                       dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                            ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4,
                                            bc=("reflective", "periodic", "periodic")), 6),
    # RK3 time stepping (TIME_STEPPING RK3)
    "mhd2d_mc_hlld_ucthlld_rk3": (ics.mhd2d_turbulence, dict(n=(28, 24), seed=91),
                                  dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                       ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4, rk="RK3"), 12),
    "mhd3d_mc_hlld_ucthlld_rk3": (ics.mhd3d_turbulence, dict(n=(12, 10, 8), seed=92),
                                  dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                       ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4, rk="RK3"), 8),
    "mhd2d_ppm_hlld_ucthlld_outflow_rk3": (
        ics.mhd2d_turbulence, dict(n=(24, 22), seed=93),
        dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
             first_dt=1e-4, reconstruction="PARABOLIC", rk="RK3",
             bc=("outflow", "outflow", "periodic")), 10),
    "hd2d_ppm_hllc_reflect_rk3": (ics.hd_turbulence, dict(n=(26, 20), seed=94),
                                  dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc",
                                       cfl=0.4, first_dt=1e-4, reconstruction="PARABOLIC",
                                       rk="RK3", bc=("reflective", "periodic", "periodic")), 12),
    "rmhd3d_mc_hlld_ucthll_rk3": (ics.rmhd3d_turbulence, dict(n=(10, 8, 8), seed=95,
                                                              lorentz_max=5.0),
                                  dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                       ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4, rk="RK3"), 6),
    # MP5 reconstruction (RECONSTRUCTION MP5, 3 ghost cells)
    "mhd2d_mp5_hlld_ucthlld": (ics.mhd2d_turbulence, dict(n=(26, 22), seed=101),
                               dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                    ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                    reconstruction="MP5"), 12),
    "mhd3d_mp5_hlld_ucthlld_rk3": (ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=102),
                                   dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                        ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                        reconstruction="MP5", rk="RK3"), 6),
    "mhd3d_blast_mp5_hll_ucthll_reflect": (
        ics.mhd3d_blast, dict(n=(14, 12, 10), seed=103, radius=0.25),
        dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hll", ct_emf="UCT_HLL", cfl=0.4,
             first_dt=1e-4, reconstruction="MP5", bc=("reflective", "outflow", "periodic")), 6),
    "hd2d_mp5_hllc": (ics.hd_turbulence, dict(n=(24, 20), seed=104),
                      dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc", cfl=0.4,
                           first_dt=1e-4, reconstruction="MP5"), 12),
    "rmhd3d_mp5_hlld_ucthll": (ics.rmhd3d_turbulence, dict(n=(10, 8, 8), seed=105,
                                                           lorentz_max=5.0),
                               dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                    ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4,
                                    reconstruction="MP5"), 6),
    # WENO-Z reconstruction (the 5-point driver of MP5, 3 ghost cells)
    "mhd2d_wenoz_hlld_ucthlld": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=141),
                                 dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                      ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                      reconstruction="WENOZ"), 10),
    "mhd3d_wenoz_hll_ucthll_outflow_rk3": (
        ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=142),
        dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hll", ct_emf="UCT_HLL", cfl=0.4,
             first_dt=1e-4, reconstruction="WENOZ", rk="RK3",
             bc=("outflow", "periodic", "periodic")), 6),
    "hd2d_wenoz_hllc_reflect": (ics.hd_turbulence, dict(n=(22, 18), seed=143),
                                dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc",
                                     cfl=0.4, first_dt=1e-4, reconstruction="WENOZ",
                                     bc=("periodic", "reflective", "periodic")), 12),
    "rmhd3d_wenoz_hlld_ucthll": (ics.rmhd3d_turbulence, dict(n=(10, 8, 8), seed=144,
                                                             lorentz_max=5.0),
                                 dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                      ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4,
                                      reconstruction="WENOZ"), 6),
    "rmhd3d_mc_tvdlf_ucthll": (ics.rmhd3d_turbulence, dict(n=(10, 8, 8), seed=165,
                                                           lorentz_max=5.0),
                               dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="tvdlf",
                                    ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4), 6),
    # CT_EMF_AVERAGE ARITHMETIC (face EMFs from the induction fluxes)
    "mhd2d_mc_hlld_arith": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=181),
                            dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                 ct_emf="ARITHMETIC", cfl=0.4, first_dt=1e-4), 12),
    "mhd3d_vl_hll_arith_outflowy": (
        ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=182),
        dict(physics="MHD", ndim=3, limiter="VANLEER_LIM", solver="hll", ct_emf="ARITHMETIC",
             cfl=0.4, first_dt=1e-4, bc=("periodic", "outflow", "periodic")), 6),
    "mhd2d_ppm_tvdlf_arith": (ics.mhd2d_turbulence, dict(n=(22, 18), seed=183),
                              dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="tvdlf",
                                   ct_emf="ARITHMETIC", cfl=0.4, first_dt=1e-4,
                                   reconstruction="PARABOLIC"), 10),
    # CT_EMF_AVERAGE CT_CONTACT (face EMFs + contact-upwinded corner terms)
    "mhd2d_mc_hlld_contact": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=201),
                              dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                   ct_emf="CT_CONTACT", cfl=0.4, first_dt=1e-4), 12),
    "mhd3d_mc_hlld_contact": (ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=202),
                              dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                   ct_emf="CT_CONTACT", cfl=0.4, first_dt=1e-4), 8),
    "mhd3d_vl_hll_contact_outflowy": (
        ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=203),
        dict(physics="MHD", ndim=3, limiter="VANLEER_LIM", solver="hll", ct_emf="CT_CONTACT",
             cfl=0.4, first_dt=1e-4, bc=("periodic", "outflow", "periodic")), 6),
    "mhd2d_ppm_hllc_contact_rk3": (ics.mhd2d_turbulence, dict(n=(22, 18), seed=204),
                                   dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hllc",
                                        ct_emf="CT_CONTACT", cfl=0.4, first_dt=1e-4,
                                        reconstruction="PARABOLIC", rk="RK3"), 10),
    "mhd3d_blast_mc_tvdlf_contact_reflect": (
        ics.mhd3d_blast, dict(n=(14, 12, 10), seed=205, radius=0.25),
        dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="tvdlf", ct_emf="CT_CONTACT",
             cfl=0.4, first_dt=1e-4, bc=("reflective", "reflective", "reflective")), 6),
    # HLLC for MHD (Src/MHD/hllc.cpp): UCT_HLL and ARITHMETIC face data
    "mhd2d_mc_hllc_ucthll": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=191),
                             dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hllc",
                                  ct_emf="UCT_HLL", cfl=0.4, first_dt=1e-4), 12),
    "mhd3d_vl_hllc_arith_outflowx": (
        ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=192),
        dict(physics="MHD", ndim=3, limiter="VANLEER_LIM", solver="hllc", ct_emf="ARITHMETIC",
             cfl=0.4, first_dt=1e-4, bc=("outflow", "periodic", "periodic")), 6),
    "mhd2d_ppm_hllc_ucthll_rk3": (ics.mhd2d_turbulence, dict(n=(22, 18), seed=193),
                                  dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hllc",
                                       ct_emf="UCT_HLL", cfl=0.4, first_dt=1e-4,
                                       reconstruction="PARABOLIC", rk="RK3"), 10),
    "mhd3d_blast_mc_hllc_ucthll_reflect": (
        ics.mhd3d_blast, dict(n=(14, 12, 10), seed=194, radius=0.25),
        dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hllc", ct_emf="UCT_HLL", cfl=0.4,
             first_dt=1e-4, bc=("reflective", "reflective", "reflective")), 8),
    # the Lax-Friedrichs (tvdlf) solver, MHD with UCT_HLL face data and HD
    "mhd2d_mc_tvdlf_ucthll": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=161),
                              dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="tvdlf",
                                   ct_emf="UCT_HLL", cfl=0.4, first_dt=1e-4), 12),
    "mhd3d_vl_tvdlf_ucthll_outflowx": (
        ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=162),
        dict(physics="MHD", ndim=3, limiter="VANLEER_LIM", solver="tvdlf", ct_emf="UCT_HLL",
             cfl=0.4, first_dt=1e-4, bc=("outflow", "periodic", "periodic")), 6),
    "hd2d_mc_tvdlf_reflect": (ics.hd_turbulence, dict(n=(22, 18), seed=163),
                              dict(physics="HD", ndim=2, limiter="MC_LIM", solver="tvdlf",
                                   cfl=0.4, first_dt=1e-4,
                                   bc=("reflective", "periodic", "periodic")), 12),
    "hd3d_ppm_tvdlf": (ics.hd_turbulence, dict(n=(12, 10, 9), seed=164),
                       dict(physics="HD", ndim=3, limiter="MC_LIM", solver="tvdlf", cfl=0.4,
                            first_dt=1e-4, reconstruction="PARABOLIC"), 8),
    # LimO3 and WENO3 (3-point stencils of the same driver, 2 ghost cells)
    "mhd2d_limo3_hlld_ucthlld": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=151),
                                 dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                                      ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                      reconstruction="LimO3"), 10),
    "mhd3d_weno3_hlld_ucthlld_outflowz": (
        ics.mhd3d_turbulence, dict(n=(12, 10, 9), seed=152),
        dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
             first_dt=1e-4, reconstruction="WENO3", bc=("periodic", "periodic", "outflow")), 6),
    "hd2d_limo3_hllc_reflect": (ics.hd_turbulence, dict(n=(22, 18), seed=153),
                                dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc",
                                     cfl=0.4, first_dt=1e-4, reconstruction="LimO3",
                                     bc=("reflective", "periodic", "periodic")), 12),
    "hd3d_weno3_hll_rk3": (ics.hd_turbulence, dict(n=(12, 10, 9), seed=154),
                           dict(physics="HD", ndim=3, limiter="MC_LIM", solver="hll", cfl=0.4,
                                first_dt=1e-4, reconstruction="WENO3", rk="RK3"), 8),
    "rmhd3d_limo3_hlld_ucthll": (ics.rmhd3d_turbulence, dict(n=(10, 8, 8), seed=155,
                                                             lorentz_max=5.0),
                                 dict(physics="RMHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                      ct_emf="UCT_HLL", cfl=0.3, first_dt=1e-4,
                                      reconstruction="LimO3"), 6),
    # the other PLM limiters of Src/plm_coeffs.hpp (uniform-grid forms)
    "mhd2d_flat_hlld_ucthlld": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=121),
                                dict(physics="MHD", ndim=2, limiter="FLAT_LIM", solver="hlld",
                                     ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4), 10),
    "mhd2d_vanalbada_hlld_ucthlld": (ics.mhd2d_turbulence, dict(n=(22, 26), seed=122),
                                     dict(physics="MHD", ndim=2, limiter="VANALBADA_LIM",
                                          solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
                                          first_dt=1e-4), 12),
    "mhd3d_ospre_hlld_ucthll": (ics.mhd3d_turbulence, dict(n=(12, 10, 14), seed=123),
                                dict(physics="MHD", ndim=3, limiter="OSPRE_LIM", solver="hlld",
                                     ct_emf="UCT_HLL", cfl=0.4, first_dt=1e-4), 8),
    "mhd2d_umist_hll_ucthll_outflow": (
        ics.mhd2d_turbulence, dict(n=(20, 18), seed=124),
        dict(physics="MHD", ndim=2, limiter="UMIST_LIM", solver="hll", ct_emf="UCT_HLL", cfl=0.4,
             first_dt=1e-4, bc=("outflow", "periodic", "periodic")), 12),
    "hd3d_umist_hllc": (ics.hd_turbulence, dict(n=(12, 14, 10), seed=125),
                        dict(physics="HD", ndim=3, limiter="UMIST_LIM", solver="hllc", cfl=0.4,
                             first_dt=1e-4), 8),
    "hd2d_ospre_hll": (ics.hd_turbulence, dict(n=(26, 20), seed=126),
                       dict(physics="HD", ndim=2, limiter="OSPRE_LIM", solver="hll", cfl=0.4,
                            first_dt=1e-4), 12),
    # USERDEF sides: the inflow rule of oracle/ref/init.cpp UserDefBoundary,
    # then the framework's div B = 0 normal faces and ghost averages
    "mhd2d_mc_hlld_ucthlld_userdefx": (ics.mhd2d_turbulence, dict(n=(24, 20), seed=111),
                                       dict(physics="MHD", ndim=2, limiter="MC_LIM",
                                            solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
                                            first_dt=1e-4,
                                            bc=("userdef", "periodic", "periodic")), 12),
    "mhd2d_ppm_hlld_ucthlld_userdefx_outflowy": (
        ics.mhd2d_turbulence, dict(n=(22, 18), seed=112),
        dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
             first_dt=1e-4, reconstruction="PARABOLIC", bc=("userdef", "outflow", "periodic")), 10),
    "mhd2d_mp5_hll_ucthll_userdefy_rk3": (
        ics.mhd2d_turbulence, dict(n=(20, 24), seed=113),
        dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hll", ct_emf="UCT_HLL", cfl=0.4,
             first_dt=1e-4, reconstruction="MP5", rk="RK3",
             bc=("periodic", "userdef", "periodic")), 10),
    "hd2d_mc_hllc_userdefy": (ics.hd_turbulence, dict(n=(20, 22), seed=114),
                              dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc",
                                   cfl=0.4, first_dt=1e-4,
                                   bc=("reflective", "userdef", "periodic")), 12),
    "mhd3d_mc_hlld_ucthlld_userdefz": (ics.mhd3d_turbulence, dict(n=(12, 10, 14), seed=115),
                                       dict(physics="MHD", ndim=3, limiter="MC_LIM",
                                            solver="hlld", ct_emf="UCT_HLLD", cfl=0.4,
                                            first_dt=1e-4,
                                            bc=("outflow", "periodic", "userdef")), 8),
}


# Output/restart cases: .dbl output every `every` steps, then a restart of
# the reference from output #1 run to step `nsteps`.
# name: (generator, kwargs, RefConfig kwargs, every, nsteps)
IO_CASES = {
    "io_mhd2d_dbl": (ics.mhd2d_turbulence, dict(n=(24, 16), seed=21),
                     dict(physics="MHD", ndim=2, limiter="MC_LIM", solver="hlld",
                          ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4), 4, 8),
    "io_mhd3d_outflowx_dbl": (ics.mhd3d_turbulence, dict(n=(12, 10, 8), seed=22),
                              dict(physics="MHD", ndim=3, limiter="MC_LIM", solver="hlld",
                                   ct_emf="UCT_HLLD", cfl=0.4, first_dt=1e-4,
                                   bc=("outflow", "periodic", "periodic")), 3, 6),
    "io_hd2d_dbl": (ics.hd_turbulence, dict(n=(20, 12), seed=23),
                    dict(physics="HD", ndim=2, limiter="MC_LIM", solver="hllc",
                         cfl=0.4, first_dt=1e-4), 3, 6),
}


def make_io(name: str) -> str:
    """Reference .dbl files of outputs #0 and #1, dbl.out, restart.out, and the
    reference's own restart from #1 run to step nsteps."""
    gen, kw, rc, every, nsteps = IO_CASES[name]
    st = gen(**kw)
    if rc["ndim"] == 2 and st.ndim == 3:
        st = _as2d(st)
    cfg = br.RefConfig(name=ref_cfg_name(rc), n=st.shape, **rc)
    binary = br.build(cfg)
    with tempfile.TemporaryDirectory() as tmp:
        icp = os.path.join(tmp, "ic.bin")
        ics.write_ic(icp, st)
        br.run_ref_io(binary, icp, every, every + 1, tmp)
        files = {f: open(os.path.join(tmp, f), "rb").read()
                 for f in ("data.0000.dbl", "data.0001.dbl", "dbl.out", "restart.out")}
        d = br.run_ref_io(binary, icp, every, nsteps, tmp, restart=1,
                          dump_path=os.path.join(tmp, "rst.dump"))
    os.makedirs(os.path.join(HERE, "io"), exist_ok=True)
    out = os.path.join(HERE, "io", f"{name}.npz")
    u8 = lambda b: np.frombuffer(b, np.uint8)
    np.savez_compressed(
        out, physics=st.physics, ndim=st.ndim, shape=np.array(st.shape), gamma=st.gamma,
        V0=st.V, Bs0=np.array(st.Bs) if st.Bs else np.zeros(0),
        dbl0=u8(files["data.0000.dbl"]), dbl1=u8(files["data.0001.dbl"]),
        dbl_out=u8(files["dbl.out"]), restart_out=u8(files["restart.out"]),
        rst_V=d.V, rst_U=d.U, rst_Bs=np.array(d.Bs) if d.Bs else np.zeros(0), rst_dt=d.dt,
        every=every, nsteps=nsteps, limiter=rc["limiter"], solver=rc["solver"],
        ct=rc.get("ct_emf", "none"), cfl=rc["cfl"], cfl_max_var=1.1, first_dt=rc["first_dt"],
        reconstruction=rc.get("reconstruction", "LINEAR"), outflow=outflow_mask(rc))
    return out


def ref_cfg_name(rc: dict) -> str:
    lim = {"PARABOLIC": "ppm", "MP5": "mp5", "WENOZ": "wenoz", "LimO3": "limo3",
           "WENO3": "weno3"}.get(rc.get("reconstruction"), rc["limiter"])
    rk = "_rk3" if rc.get("rk") == "RK3" else ""
    return "{physics}{ndim}d_{lim}_{solver}_{ct}".format(
        ct=rc.get("ct_emf", "none"), lim=lim, **rc).lower() + rk


def _as2d(st):
    """Take the first z-plane of a 3-D state as a 2-D state (Bz cell-centred)."""
    V = st.V[:, :1].copy()
    Bs = [st.Bs[0][:1].copy(), st.Bs[1][:1].copy()]
    V[ics.BX1] = 0.5 * (Bs[0] + np.roll(Bs[0], -1, axis=2))
    V[ics.BX2] = 0.5 * (Bs[1] + np.roll(Bs[1], -1, axis=1))
    return ics.PrimState(st.physics, 2, (st.shape[0], st.shape[1], 1), st.gamma, V, Bs)


def side_mask(rc: dict, kinds=("outflow",)) -> int:
    """Bits 2d and 2d+1 set for each direction d whose sides are of `kinds`."""
    m = 0
    for d, t in enumerate(rc.get("bc", ("periodic",) * 3)):
        if t in kinds and d < rc["ndim"]:
            m |= 3 << (2 * d)
    return m


def outflow_mask(rc: dict) -> int:
    return side_mask(rc, ("outflow",))


def make(name: str) -> str:
    gen, kw, rc, nsteps = CASES[name]
    st = gen(**kw)
    if rc["ndim"] == 2 and st.ndim == 3:
        st = _as2d(st)
    cfg = br.RefConfig(name=ref_cfg_name(rc), n=st.shape, **rc)
    # the grid size is a run-time ini parameter: one binary per scheme,
    # re-using objects; the ini is rewritten per case
    binary = br.build(cfg)
    with tempfile.TemporaryDirectory() as tmp:
        icp = os.path.join(tmp, "ic.bin")
        dmp = os.path.join(tmp, "out.dump")
        ics.write_ic(icp, st)
        d = br.run_ref(binary, icp, nsteps, dmp)
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(
        out, physics=st.physics, ndim=st.ndim, shape=np.array(st.shape), gamma=st.gamma,
        V0=st.V, Bs0=np.array(st.Bs) if st.Bs else np.zeros(0),
        V=d.V, U=d.U, Bs=np.array(d.Bs) if d.Bs else np.zeros(0), dt=d.dt, nsteps=nsteps,
        limiter=rc["limiter"], solver=rc["solver"], ct=rc.get("ct_emf", "none"),
        cfl=rc["cfl"], cfl_max_var=1.1, first_dt=rc["first_dt"],
        reconstruction=rc.get("reconstruction", "LINEAR"), outflow=outflow_mask(rc),
        reflect=side_mask(rc, ("reflective", "axisymmetric")),
        eqtsym=side_mask(rc, ("eqtsymmetric",)), userdef=side_mask(rc, ("userdef",)),
        rk=3 if rc.get("rk") == "RK3" else 2)
    return out


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES) + list(IO_CASES)
    for nm in names:
        p = make_io(nm) if nm in IO_CASES else make(nm)
        print(f"{nm}: {os.path.getsize(p)/1024:.0f} KiB")
