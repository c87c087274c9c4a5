"""The FEAT3-side shim (feat3_b200/shim/feat_arch_cuda.cpp), compiled against the reference's own
kernel/lafem/arch headers, binds LAFEM::Arch::<Op><Mem::CUDA> onto libfeat3_b200. The check
program tests/shim/shim_check.cpp (built by `make -C oracle shim`, which needs the reference's
sources, so it is built ahead and run here from oracle/_ref/) calls the reference's declarations
-- Apply::csr for both index types (apply.hpp:271-275) and transposed, Apply::ell
(apply.hpp:296), Axpy, DotProduct, Norm2, ComponentProduct, ComponentInvert, Scale, Diagonal and
UnitFilter -- on cudaMalloc'd buffers and compares each result with the reference's own
Mem::Main templates (kernel/lafem/arch/*_generic.hpp) on the same inputs."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK = os.path.join(ROOT, "oracle", "_ref", "shim_check")


def test_shim_check_links_against_the_library():
    if not os.path.exists(CHECK):
        pytest.skip("oracle/_ref/shim_check was not built (the reference sources were absent at build time)")
    out = subprocess.run(["ldd", CHECK], capture_output=True, text=True).stdout
    assert "libfeat3_b200.so" in out and "not found" not in out, out


@pytest.mark.gpu
def test_reference_arch_declarations_run_on_the_library():
    if not os.path.exists(CHECK):
        pytest.skip("oracle/_ref/shim_check was not built (the reference sources were absent at build time)")
    res = subprocess.run([CHECK], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    lines = res.stdout.splitlines()
    assert lines[-1].startswith("PASSED"), res.stdout
    for tag in ("f64/u32 csr", "f64/u64 csr", "f32/u64 csr", "f64/u64 csr^T", "f64/u64 ell", "f64/u64 diagonal csr",
                "f64/u64 unit filter rhs", "f64 dot", "f64 norm2", "invalid arguments -> InternalError"):
        assert any(l.startswith("ok " + tag) for l in lines), (tag, res.stdout)
