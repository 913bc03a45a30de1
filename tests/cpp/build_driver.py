"""Builds tests/cpp/_build/dropin_driver: the C++ drop-in module driven like
the reference's example drivers, on the stand-in coupler of oracle/ref_shim
(which includes the reference's MultipleFields.h, so the build needs the
reference tree; the GPU box uses the binary built here)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(HERE, "_build", "dropin_driver")
PHYS_EXE = os.path.join(HERE, "_build", "physics_driver")
PG_EXE = os.path.join(HERE, "_build", "pg_driver")
# The reference tree: $PORTURB_REFERENCE, by default where this image mounts it.
REF_CORE = os.path.join(os.environ.get("PORTURB_REFERENCE", "/root/reference"), "model", "core")


def _compile(src, exe, libdir):
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "porturb_b200", "cpp"),
           "-I", os.path.join(ROOT, "oracle", "ref_shim"), "-I", os.path.join(ROOT, "include"), "-I", REF_CORE,
           os.path.join(HERE, src), "-o", exe, "-L", libdir, "-lpu_dycore", "-Wl,-rpath," + libdir]
    subprocess.run(cmd, check=True)


def build(libdir):
    """Builds the drivers (the dycore drop-in alone, the boundary-layer module
    chain, the pressure-gradient forcings); returns the dycore driver's path, or None without the
    reference tree and without a prebuilt binary."""
    if not os.path.isdir(REF_CORE):
        return EXE if os.path.exists(EXE) else None
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    _compile("dropin_driver.cpp", EXE, libdir)
    _compile("physics_driver.cpp", PHYS_EXE, libdir)
    _compile("pg_driver.cpp", PG_EXE, libdir)
    return EXE
