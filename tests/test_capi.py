"""CPU-side checks of the C-ABI library: it loads, and it exports every symbol that
include/feat3_b200.h declares (no compute call is made without a GPU)."""
import ctypes
import subprocess

from feat3_b200 import _lib, build


def test_library_builds_and_loads():
    lib = _lib.load()
    assert lib.fb_version().decode().startswith("feat3_b200")


def test_every_header_symbol_is_exported():
    syms = _lib.header_symbols()
    assert len(syms) >= 40
    lib = ctypes.CDLL(build.LIB)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert set(syms) <= exported
    # nothing but the declared C-ABI is exported under the fb_ prefix
    assert {s for s in exported if s.startswith("fb_")} == set(syms)


def test_every_header_symbol_has_a_binding():
    assert set(_lib.header_symbols()) == set(_lib._SIGS)


def test_invalid_arguments_are_rejected_without_a_gpu():
    lib = _lib.load()
    # null pointers / bad sizes are caught on the host before any CUDA call
    assert lib.fb_axpy_f64(None, 1.0, None, None, 10, None) == _lib.FB_ERR_INVALID
    assert lib.fb_csr_apply_f64(None, 1.0, None, 1.0, None, None, None, None, 5, 5, 5, 0, None) == _lib.FB_ERR_INVALID
    assert lib.fb_mg_create_structured(None, None) == _lib.FB_ERR_INVALID
    h = ctypes.c_void_p()
    bad = _lib.StructuredDesc(4, 1, 3, 1, None, 0, 1, 0)
    assert lib.fb_mg_create_structured(ctypes.byref(h), ctypes.byref(bad)) == _lib.FB_ERR_INVALID
    cfg = _lib.SolverCfg()
    lib.fb_solver_cfg_default(ctypes.byref(cfg))
    assert (cfg.outer, cfg.nu, cfg.coarse, cfg.precision) == (0, 4, 0, 0)
    assert abs(cfg.tol_rel - 1e-8) < 1e-20 and abs(cfg.omega_jac - 0.5) < 1e-15
    assert lib.fb_mg_configure(None, ctypes.byref(cfg)) == _lib.FB_ERR_INVALID


def test_plain_c_client_of_the_io_entry_points(tmp_path):
    """the header compiles as C99 and a C program linked against the library round-trips the
    reference's own files through fb_io_* (host code, no GPU)"""
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    exe = tmp_path / "io_client"
    libdir = os.path.dirname(build.LIB)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I" + os.path.join(root, "include"),
                    os.path.join(here, "capi_client", "io_client.c"), "-o", str(exe), "-L" + libdir, "-lfeat3_b200",
                    "-Wl,-rpath," + libdir], check=True)
    files = os.path.join(here, "golden", "feat_files_q1_2d_L3")
    out = subprocess.run([str(exe), os.path.join(files, "L3.A.csr"), os.path.join(files, "rhs.dv"), str(tmp_path)],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert "matrix 81 x 81, 625 entries" in out.stdout and "vector 81 values" in out.stdout
