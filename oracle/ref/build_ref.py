"""Build and run the reference gPLUTO serial CPU binary as a parity checker.

Test infrastructure only.  For one scheme configuration this writes a
``definitions.hpp``, a ``pluto.ini`` and a short Makefile of our own into
``oracle/_ref/<name>/`` and compiles the reference sources in place under
``$GP_REFERENCE_ROOT/Src`` (never copied; by default the ``reference``
directory beside this repository) together with ``oracle/ref/init.cpp``,
using the flags of the reference's serial build ``Config/linux.g++.defs``
(``g++ -O3 -std=c++17``).  The object lists follow
``Src/Templates/default_objects.mk``, ``Src/MHD/makefile``,
``Src/MHD/CT/makefile``, ``Src/HD/makefile`` and ``Src/RMHD/makefile``.

``run_ref`` executes the binary on a seeded IC file with FTZ/DAZ disabled
(``GPLUTO_FTZ_DAZ=0``, ``Src/cpu_fp.hpp:11-16``; the GPU never flushes
denormals) and reads back the state dumped by ``init.cpp`` after N steps.
"""
from __future__ import annotations

import dataclasses
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.path.abspath(os.environ.get(
    "GP_REFERENCE_ROOT", os.path.join(HERE, "..", "..", "..", "reference")))
OUT_ROOT = os.path.join(os.path.dirname(HERE), "_ref")

_DEFAULT_OBJ = """arrays array_reconstruct bin_io boundary cmd_line_opt data2sweep
debug_tools euler_step fallback flag_boundary flag_exchange flag_shock flat_states
get_nghost globals init initialize input_data internal_boundary jet_domain main
mapped_grid_tools mappers3D mean_mole_weight mem_usage next_time_step nvtx
output_grid output_log parallel_exchange_async parallel_exchange_sync parse_file
rbox ring_average ring_average_rec restart rotate runtime_setup source
set_geometry set_grid set_output set_var_names show_config split_source startup
sweep_alloc timing tools write_data write_tab write_vtk vector_curl
userdef_output""".split()
_MATH_OBJ = "math_lu_decomp math_funcs math_misc math_quadrature math_random".split()
_STEP_OBJ = "plm_states rk_step update_stage".split()   # ppm_states for PARABOLIC
_PHYS = {
    "MHD": ("mappers roe set_solver tvdlf hlld hll hllc rhs gforce".split(),
            ["MHD"]),
    "HD": ("mappers hll hllc rhs roe set_solver tvdlf two_shock".split(),
           ["HD", "MHD"]),
    "RMHD": ("""pcp_nr pcp_stage rmhd_consistency mappers set_solver hll hllc hlld
rmhd_energy_solve rmhd_pressure_fix rmhd_entropy_solve tvdlf rhs gforce""".split(),
             ["RMHD", "RHD"]),
}
_CT_OBJ = """ct_field_average ct_emf ct_emf_average ct_eng_correction
ct_imex_update_ELR ct_maxwell_solver ct_update ct_fill_mag_field""".split()


@dataclasses.dataclass
class RefConfig:
    name: str
    physics: str = "MHD"          # MHD | HD | RMHD
    ndim: int = 2
    n: tuple = (32, 32, 1)
    limiter: str = "MC_LIM"       # MC_LIM | VANLEER_LIM | MINMOD_LIM
    solver: str = "hlld"          # hlld | hll | hllc
    ct_emf: str = "UCT_HLLD"      # UCT_HLLD | UCT_HLL (MHD/RMHD only)
    rk: str = "RK2"
    cfl: float = 0.4
    cfl_max_var: float = 1.1
    first_dt: float = 1.0e-4
    reconstruction: str = "LINEAR"
    bc: tuple = ("periodic", "periodic", "periodic")   # per direction, both sides

    def definitions(self) -> str:
        lines = [
            f"#define  PHYSICS                 {self.physics}",
            f"#define  DIMENSIONS              {self.ndim}",
            "#define  GEOMETRY                CARTESIAN",
            "#define  MAPPED_GRID             NO",
            "#define  BODY_FORCE              NO",
            "#define  COOLING                 NO",
            f"#define  RECONSTRUCTION          {self.reconstruction}",
            f"#define  TIME_STEPPING           {self.rk}",
            "#define  NTRACER                 0",
            "#define  PARTICLES               NO",
            "#define  USER_DEF_PARAMETERS     0",
            "#define  EOS                     IDEAL",
            "#define  ENTROPY_SWITCH          NO",
        ]
        if self.physics in ("MHD", "RMHD"):
            lines += [
                "#define  DIVB_CONTROL            CONSTRAINED_TRANSPORT",
                "#define  BACKGROUND_FIELD        NO",
                f"#define  CT_EMF_AVERAGE          {self.ct_emf}",
                "#define  CT_ENERGY_CORRECTION    NO",
                "#define  ASSIGN_VECTOR_POTENTIAL NO",
            ]
        if self.physics == "MHD":
            lines += ["#define  AMBIPOLAR_DIFFUSION     NO",
                      "#define  RESISTIVITY             NO",
                      "#define  HALL_MHD                NO"]
        if self.physics == "RMHD":
            lines += ["#define  RESISTIVITY             NO"]
        if self.physics in ("HD", "MHD"):
            lines += ["#define  THERMAL_CONDUCTION      NO",
                      "#define  VISCOSITY               NO"]
        lines += ["#define  ROTATING_FRAME          NO",
                  f"#define  LIMITER                 {self.limiter}",
                  "#define  WARNING_MESSAGES        0"]
        return "\n".join(lines) + "\n"

    def ini(self) -> str:
        nx, ny, nz = self.n
        g = [f"X1-grid    0.0  {nx}  1.0",
             f"X2-grid    0.0  {ny if self.ndim >= 2 else 1}  1.0",
             f"X3-grid    0.0  {nz if self.ndim == 3 else 1}  1.0"]
        return "\n".join([
            "[Grid]", "", *g, "",
            "[Time]", "",
            f"CFL              {self.cfl!r}",
            f"CFL_max_var      {self.cfl_max_var!r}",
            "tstop            1.e30",
            f"first_dt         {self.first_dt!r}", "",
            "[Solver]", "", f"Solver           {self.solver}", "",
            "[Boundary]", "",
            *[f"X{d}-{s}        {self.bc[d - 1]}" for d in (1, 2, 3) for s in ("beg", "end")], "",
            "[Static Grid Output]", "",
            "uservar    0",
            "dbl       -1.0  -1   single_file",
            "flt       -1.0  -1   single_file",
            "vtk       -1.0  -1   single_file",
            "dbl.h5    -1.0  -1",
            "flt.h5    -1.0  -1",
            "tab       -1.0  -1",
            "ppm       -1.0  -1",
            "png       -1.0  -1",
            "log        1000000000",
            "analysis  -1.0   1", "",
            "[Particles]", "",
            "Nparticles          -1     1",
            "particles_dbl       -1.0  -1",
            "particles_flt       -1.0  -1",
            "particles_vtk       -1.0  -1",
            "particles_tab       -1.0  -1", "",
            "[Parameters]", "",
        ]) + "\n"

    def makefile(self) -> str:
        src = os.path.join(REF_ROOT, "Src")
        phys_obj, phys_dirs = _PHYS[self.physics]
        states = {"PARABOLIC": "ppm_states", "MP5": "mp5_states", "WENOZ": "mp5_states",
                  "LimO3": "mp5_states", "WENO3": "mp5_states"}.get(self.reconstruction,
                                                                    "plm_states")
        step = [(states if o == "plm_states" else o) for o in _STEP_OBJ]
        objs = _DEFAULT_OBJ + _MATH_OBJ + step + phys_obj
        vdirs = [src, f"{src}/States", f"{src}/Math_Tools"] + [f"{src}/{d}" for d in phys_dirs]
        incs = ["-I.", f"-I{src}"] + [f"-I{src}/{d}" for d in phys_dirs] + [f"-I{src}/States", f"-I{src}/Math_Tools"]
        if self.physics in ("MHD", "RMHD"):
            objs += _CT_OBJ
            vdirs.append(f"{src}/MHD/CT")
            incs.append(f"-I{src}/MHD/CT")
        # init.cpp comes from oracle/ref (ours); every other source from the reference tree
        vdirs.insert(0, HERE)
        uniq = []
        for o in objs:
            if o not in uniq:
                uniq.append(o)
        return "\n".join([
            "CC      = g++",
            "CFLAGS  = -c -O3 -std=c++17",
            "LDFLAGS = -lm",
            f"VPATH   = {':'.join(vdirs)}",
            f"INCS    = {' '.join(incs)}",
            f"OBJ     = {' '.join(o + '.o' for o in uniq)}",
            "",
            "pluto: $(OBJ)",
            "\t$(CC) $(OBJ) $(LDFLAGS) -o $@",
            "",
            "%.o: %.cpp definitions.hpp",
            "\t$(CC) $(CFLAGS) $(INCS) $< -o $@",
            "",
        ])


def build(cfg: RefConfig, jobs: int = 8, quiet: bool = True) -> str:
    """Compile the reference binary for ``cfg``; returns the binary path."""
    if not os.path.isdir(os.path.join(REF_ROOT, "Src")):
        raise FileNotFoundError(f"reference sources not found under {REF_ROOT}")
    d = os.path.join(OUT_ROOT, cfg.name)
    os.makedirs(d, exist_ok=True)
    for fname, text in (("definitions.hpp", cfg.definitions()),
                        ("pluto.ini", cfg.ini()),
                        ("Makefile", cfg.makefile())):
        p = os.path.join(d, fname)
        old = open(p).read() if os.path.exists(p) else None
        if old != text:
            with open(p, "w") as fh:
                fh.write(text)
    out = subprocess.run(["make", f"-j{jobs}"], cwd=d, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"reference build failed in {d}:\n{out.stdout[-4000:]}\n{out.stderr[-4000:]}")
    if not quiet:
        print(out.stdout[-2000:])
    return os.path.join(d, "pluto")


@dataclasses.dataclass
class RefDump:
    physics: int
    ndim: int
    shape: tuple
    dt: np.ndarray        # dt of each step taken (len nsteps) + the next dt
    time: np.ndarray
    wall: np.ndarray      # wall-clock stamp at the start of each step (s)
    V: np.ndarray
    U: np.ndarray
    Bs: list


def read_dump(path: str) -> RefDump:
    buf = open(path, "rb").read()
    assert buf[:4] == b"GPDM", "bad dump magic"
    ver, phys, ndim, nx, ny, nz, nvar, nh = struct.unpack_from("<8i", buf, 4)
    off = 36
    arr = lambda n: np.frombuffer(buf, "<f8", n, off)
    dt = arr(nh).copy(); off += 8 * nh
    tm = arr(nh).copy(); off += 8 * nh
    wall = arr(nh).copy(); off += 8 * nh
    nc = nx * ny * nz
    V = arr(nvar * nc).reshape(nvar, nz, ny, nx).copy(); off += 8 * nvar * nc
    U = arr(nvar * nc).reshape(nvar, nz, ny, nx).copy(); off += 8 * nvar * nc
    Bs = []
    if phys != 0:
        for _ in range(ndim):
            Bs.append(arr(nc).reshape(nz, ny, nx).copy()); off += 8 * nc
    return RefDump(phys, ndim, (nx, ny, nz), dt, tm, wall, V, U, Bs)


def run_ref(binary: str, ic_path: str, nsteps: int, dump_path: str,
            timeout: float | None = None) -> RefDump:
    """Run ``nsteps`` steps of the reference on an IC file; return its dump."""
    binary = os.path.abspath(binary)
    d = os.path.dirname(binary)
    env = dict(os.environ, GPLUTO_FTZ_DAZ="0", GP_IC_FILE=os.path.abspath(ic_path),
               GP_DUMP_STEP=str(nsteps), GP_DUMP_FILE=os.path.abspath(dump_path))
    out = subprocess.run([binary, "-no-write", "-maxsteps", str(nsteps)], cwd=d, env=env,
                         capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0 or not os.path.exists(dump_path):
        raise RuntimeError(f"reference run failed (rc={out.returncode}):\n{out.stdout[-3000:]}\n{out.stderr[-2000:]}")
    return read_dump(dump_path)


def run_ref_io(binary: str, ic_path: str, every: int, nsteps: int, workdir: str,
               restart: int | None = None, dump_path: str | None = None,
               timeout: float | None = None) -> RefDump | None:
    """Run the reference with .dbl output every ``every`` steps into ``workdir``
    (data.NNNN.dbl, dbl.out, restart.out), optionally restarting from output
    #``restart`` found there; stop at step ``nsteps`` and return the state
    dumped at that step (or None without ``dump_path``)."""
    binary = os.path.abspath(binary)
    ini = open(os.path.join(os.path.dirname(binary), "pluto.ini")).read()
    ini = ini.replace("dbl       -1.0  -1   single_file",
                      f"dbl       -1.0  {every}   single_file\noutput_dir {workdir}")
    ip = os.path.join(workdir, "pluto.ini")
    with open(ip, "w") as f:
        f.write(ini)
    env = dict(os.environ, GPLUTO_FTZ_DAZ="0", GP_IC_FILE=os.path.abspath(ic_path),
               GP_DUMP_STEP=str(nsteps), GP_DUMP_FILE=os.path.abspath(dump_path or
                                                                     os.path.join(workdir, "x.dump")))
    cmd = [binary, "-i", ip, "-maxsteps", str(nsteps)]
    if restart is not None:
        cmd += ["-restart", str(restart)]
    out = subprocess.run(cmd, cwd=workdir, env=env, capture_output=True, text=True,
                         timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"reference run failed (rc={out.returncode}):\n{out.stdout[-3000:]}")
    return read_dump(dump_path) if dump_path else None


if __name__ == "__main__":
    cfg = RefConfig(name=sys.argv[1] if len(sys.argv) > 1 else "mhd2d_mc_hlld")
    print(build(cfg, quiet=False))
