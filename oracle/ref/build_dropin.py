"""Build the reference driver with its time step on the B200 library.

Test infrastructure: the C++ caller of the C ABI that INTEGRATION.md
describes, compiled for real.  For one scheme configuration this writes,
into ``oracle/_ref/dropin_<name>/``:

* the ``definitions.hpp``, ``pluto.ini`` and object list of
  ``build_ref.RefConfig`` (the reference's serial build, ``g++ -O3``);
* ``main.cpp``: a copy of the reference's ``Src/main.cpp`` with two edits,
  made by exact text substitution (the build fails if either anchor is
  missing): ``GP_DropIn_Init(&data, &grid, &runtime, &run_config)`` before
  the main loop (``while (last_step!=1){``) and
  ``GP_DropIn_Step(&data, &grid, &Dts)`` in place of
  ``AdvanceStep (&data, &grid, &Dts)`` (``Src/main.cpp:446``);

then compiles it with every other source taken from the reference tree in
place, plus ``oracle/ref/gp_dropin.cpp`` (ours), and links
``gpluto_dev_b200/_build/libgpluto_b200.so`` (run-time path relative to the
binary).  The copy of main.cpp stays in the git-ignored build directory.

``run_dbl`` runs a binary (this one or the plain reference build) on a
seeded initial condition with ``.dbl`` output every ``every`` steps and
returns the output files' bytes.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

import build_ref as br  # noqa: E402

LIB_DIR = os.path.join(ROOT, "gpluto_dev_b200", "_build")
INC_DIR = os.path.join(ROOT, "include")

_INIT_ANCHOR = "  while (last_step!=1){\n"
_STEP_ANCHOR = "    AdvanceStep (&data, &grid, &Dts);\n"
_PROTOS = ("\nvoid GP_DropIn_Init(Data *, Grid *, Runtime *, RunConfig *);\n"
           "void GP_DropIn_Step(Data *, Grid *, timeStep *);\n")


def patched_main() -> str:
    src = open(os.path.join(br.REF_ROOT, "Src", "main.cpp")).read()
    for anchor in (_INIT_ANCHOR, _STEP_ANCHOR):
        if src.count(anchor) != 1:
            raise RuntimeError(f"anchor {anchor.strip()!r} not found once in Src/main.cpp")
    inc = '#include "gpluto.hpp"\n'
    if src.count(inc) != 1:
        raise RuntimeError("cannot place the prototypes in Src/main.cpp")
    src = src.replace(inc, inc + _PROTOS, 1)
    src = src.replace(_INIT_ANCHOR, "  GP_DropIn_Init (&data, &grid, &runtime, &run_config);\n"
                      + _INIT_ANCHOR, 1)
    src = src.replace(_STEP_ANCHOR, "    GP_DropIn_Step (&data, &grid, &Dts);\n", 1)
    return src


def makefile(cfg: "br.RefConfig") -> str:
    mk = cfg.makefile()
    lines = []
    for line in mk.splitlines():
        if line.startswith("OBJ "):
            line += " gp_dropin.o"
        elif line.startswith("INCS "):
            line += f" -I{INC_DIR}"
        elif line.startswith("LDFLAGS "):
            # run-time path relative to the binary (oracle/_ref/<dir>/pluto),
            # so that the driver finds the library wherever the tree is copied
            line = (f"LDFLAGS = -L{LIB_DIR} -lgpluto_b200 "
                    "-Wl,-rpath,'$$ORIGIN/../../../gpluto_dev_b200/_build' -lm")
        lines.append(line)
    return "\n".join(lines) + "\n"


def build(cfg: "br.RefConfig", jobs: int = 8) -> str:
    """Compile the drop-in driver for ``cfg``; returns the binary path."""
    if not os.path.isdir(os.path.join(br.REF_ROOT, "Src")):
        raise FileNotFoundError(f"reference sources not found under {br.REF_ROOT}")
    if not os.path.exists(os.path.join(LIB_DIR, "libgpluto_b200.so")):
        raise FileNotFoundError("build the library first (python -m gpluto_dev_b200.build)")
    d = os.path.join(br.OUT_ROOT, "dropin_" + cfg.name)
    os.makedirs(d, exist_ok=True)
    for fname, text in (("definitions.hpp", cfg.definitions()), ("pluto.ini", cfg.ini()),
                        ("Makefile", makefile(cfg)), ("main.cpp", patched_main())):
        p = os.path.join(d, fname)
        old = open(p).read() if os.path.exists(p) else None
        if old != text:
            with open(p, "w") as fh:
                fh.write(text)
    out = subprocess.run(["make", f"-j{jobs}"], cwd=d, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"drop-in build failed in {d}:\n{out.stdout[-4000:]}\n"
                           f"{out.stderr[-4000:]}")
    return os.path.join(d, "pluto")


def run_dbl(binary: str, ic_path: str, every: int, nsteps: int, workdir: str,
            timeout: float | None = None) -> dict:
    """Run ``binary`` from the initial condition for ``nsteps`` steps with
    .dbl output every ``every`` steps into ``workdir``; return the bytes of
    every data.NNNN.dbl, dbl.out and restart.out written there."""
    br.run_ref_io(binary, ic_path, every, nsteps, workdir, timeout=timeout)
    files = {}
    for f in sorted(os.listdir(workdir)):
        if f.startswith("data.") and f.endswith(".dbl") or f in ("dbl.out", "restart.out"):
            files[f] = open(os.path.join(workdir, f), "rb").read()
    return files
