"""Generate the golden fixtures of tests/golden/ from the REFERENCE's own solver.

Runs oracle/_ref/feat_ref (FEAT3's CPU multigrid, compiled from the reference sources by
oracle/Makefile; see oracle/ref_harness/feat_ref_driver.cpp) on small cases of every
configuration this project measures and stores its outputs, mapped to the lexicographic
lattice numbering through the DOF coordinates, as compressed .npz files:

    python tests/golden/gen_golden.py          # needs oracle/_ref/feat_ref
    python tests/golden/gen_golden.py --cycles # only the F/W-cycle and adaptive-CGC fixtures
    python tests/golden/gen_golden.py --files  # only the container-file fixtures (feat_files_q1_2d_L3/)
    python tests/golden/gen_golden.py --numbering  # only FEAT's DOF and cell numbering (ref_numbering.npz)

Inputs that are random (coefficient fields, target noise) are drawn here with numpy's
seeded generator and stored in the fixture next to the outputs.
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402


def save(name, **arrays):
    fn = os.path.join(HERE, name + ".npz")
    np.savez_compressed(fn, **arrays)
    print(f"{fn}: {os.path.getsize(fn) / 1024:.1f} KiB")


def run(name, dim, degree, level, level_min, rhs, k=None, keep_u=True, **kw):
    R = po.run_ref(dim, degree, level, level_min, rhs=rhs, k=k, **kw)
    info = R["info"]
    arrays = dict(dim=dim, degree=degree, level=level, level_min=level_min, rhs_kind=rhs,
                  iters=info["iters"], status=info["status"], hist=info["hist"],
                  rhs_checksum=np.array([R["rhs"].sum(), np.abs(R["rhs"]).sum(), (R["rhs"] ** 2).sum()]),
                  cfg=repr({k_: v for k_, v in kw.items() if k_ != "target"}))
    if keep_u:
        arrays["u"] = R["u"]
    if k is not None:
        arrays["k"] = k
    for key in ("grad", "lambda"):
        if key in R:
            arrays[key] = R[key]
    if "J" in info:
        arrays["J"] = info["J"]
    save(name, **arrays)
    return R


def cycles():
    """F and W cycles and the adaptive coarse-grid corrections (multigrid.hpp:1354-1519, 1898-1925)"""
    rng = np.random.default_rng(20261204)
    run("ref_cycle_f_q1_2d_L6", 2, 1, 6, 1, "sine", solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8,
        cycle="f")
    k4 = np.exp(rng.standard_normal(16 ** 3))
    run("ref_cycle_w_q1_3d_L4", 3, 1, 4, 1, "one", k=k4, solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8,
        cycle="w")
    run("ref_cgc_energy_q1_2d_L6", 2, 1, 6, 1, "sine", solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8,
        cgc="energy")
    k6 = np.exp(0.5 * rng.standard_normal(64 * 64))
    run("ref_cgc_defect_f_q1_2d_L6", 2, 1, 6, 1, "one", k=k6, solver="pcg", nu=2, omega_jac=0.5, coarse="direct",
        tol=1e-8, cycle="f", cgc="defect")
    run("ref_cycle_w_richardson_q1_2d_L5", 2, 1, 5, 1, "sine", solver="richardson", nu=3, omega_jac=0.5,
        omega_rich=1.0, coarse="smoother", tol=1e-8, cycle="w")


def feat_files():
    """The hierarchy of the 2D Q1 level-3 case (levels 3..1) as written by the reference's own
    SparseMatrixCSR/DenseVector/SparseVector::write_out (sparse_matrix_csr.hpp:1261-1343,
    dense_vector.hpp:721-777, sparse_vector.hpp:639-680; the filters' Dirichlet lists), and the
    reference's own parse of its text files written back in binary (*.mtx.csr,
    *.exp.dv, *.vmtx.dv; read_from, sparse_matrix_csr.hpp:1098-1246, dense_vector.hpp:587-712)."""
    R = po.run_ref(2, 1, 3, 1, rhs="sine", solver="pcg", nu=2, coarse="direct", tol=1e-8, feat_files=True)
    pre = R["prefix"]
    out = os.path.join(HERE, "feat_files_q1_2d_L3")
    os.makedirs(out, exist_ok=True)
    names = [f"L{l}.A.csr" for l in (1, 2, 3)] + [f"L{l}.{m}.csr" for l in (2, 3) for m in "PR"]
    names += ["L3.A.mtx", "L3.A.sym.mtx", "L3.A.mtx.csr", "L3.A.sym.mtx.csr", "L3.P.mtx", "L3.R.mtx"]
    names += [f"L{l}.filter.mtx" for l in (1, 2, 3)]
    names += ["rhs.dv", "rhs.exp", "rhs.vmtx", "rhs.exp.dv", "rhs.vmtx.dv", "u.dv"]
    total = 0
    for nm in names:
        shutil.copyfile(f"{pre}.{nm}", os.path.join(out, nm))
        total += os.path.getsize(os.path.join(out, nm))
    with open(os.path.join(out, "iters.txt"), "w") as f:
        f.write(f"{R['info']['iters']}\n")
    print(f"{out}: {len(names)} files, {total / 1024:.1f} KiB")


def numbering():
    """FEAT's own DOF and cell numbering of the refined unit square / cube, per level, as the
    lexicographic lattice index of each FEAT DOF (from its interpolated coordinates) and of each
    FEAT cell (from its centroid)"""
    arrays = {}
    for dim, degree, lmax in ((2, 1, 5), (2, 2, 4), (3, 1, 4), (3, 2, 3)):
        R = po.run_ref(dim, degree, lmax, 1, rhs="sine", solver="pcg", nu=2, coarse="direct", tol=1e-6,
                       dump_matrices=True)
        pre = R["prefix"]
        for l in range(1, lmax + 1):
            arrays[f"d{dim}_q{degree}_L{l}_dofs"] = np.fromfile(f"{pre}.L{l}.lattice", dtype=np.uint64).astype(np.uint32)
            arrays[f"d{dim}_q{degree}_L{l}_cells"] = np.fromfile(f"{pre}.L{l}.cells", dtype=np.uint64).astype(np.uint32)
    save("ref_numbering", **arrays)


def main():
    if not po.have_ref():
        sys.exit("oracle/_ref/feat_ref is missing: build it with `make -C oracle ref` first")
    if "--cycles" in sys.argv:
        return cycles()
    if "--files" in sys.argv:
        return feat_files()
    if "--numbering" in sys.argv:
        return numbering()
    rng = np.random.default_rng(20261203)
    # applications/poisson_dirichlet.cpp composition, level 5, the reference's pin (4 +- 1 iterations,
    # applications/CMakeLists.txt:100-108)
    run("ref_poisson_dirichlet_L5", 2, 1, 5, 0, "expbubble", solver="pcg", nu=4, omega_jac=0.7, omega_rich=1.0,
        coarse="smoother", tol=1e-8)
    # tutorials/tutorial_05_multigrid.cpp composition, level 7 (Richardson(MG), PCG coarse solver)
    run("ref_tutorial05_L7", 2, 1, 7, 1, "sine", solver="richardson", nu=4, omega_jac=1.0, omega_rich=0.8,
        coarse="pcg", tol=float(np.sqrt(np.finfo(np.float64).eps)), max_iter=100, keep_u=False)
    # configuration shapes (2D Q1 full size; the others reduced so the CPU oracle runs in seconds)
    run("ref_c1_q1_2d_L7", 2, 1, 7, 1, "sine", solver="pcg", nu=4, omega_jac=0.5, coarse="direct", tol=1e-8)
    run("ref_c2_q1_3d_L4", 3, 1, 4, 1, "sine", solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
    k3 = np.exp(rng.standard_normal(32 * 32))
    run("ref_c3_q2_2d_L5", 2, 2, 5, 1, "one", k=k3, solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
    k5 = np.exp(rng.standard_normal(16 ** 3))
    run("ref_c5_q1_3d_L4", 3, 1, 4, 1, "one", k=k5, solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
    kq2 = np.exp(rng.standard_normal(8 ** 3))
    run("ref_q2_3d_L3", 3, 2, 3, 1, "one", k=kq2, solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
    # mixed precision: FP64 Richardson around ConvertPrecond(FP32 MG) and the FP16-quantised variant
    for inner in ("f32", "f16"):
        run(f"ref_mixed_{inner}_q1_3d_L4", 3, 1, 4, 1, "one", k=k5, solver="richardson", nu=2, omega_jac=0.5,
            coarse="direct", tol=1e-8, inner=inner)
    # adjoint: 2D Q1, k = exp(g), g ~ N(0, 0.25) read as variance (sigma 0.5); u_target = u(k=1) + noise
    lvl = 6
    g = 0.5 * rng.standard_normal((1 << lvl) ** 2)
    u1 = po.run_ref(2, 1, lvl, 1, rhs="one", solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-14)["u"]
    target = u1 + 1e-2 * rng.standard_normal(u1.size)
    R = run("ref_adjoint_q1_2d_L6", 2, 1, lvl, 1, "one", k=np.exp(g), target=target, solver="pcg", nu=2,
            omega_jac=0.5, coarse="direct", tol=1e-14)
    fn = os.path.join(HERE, "ref_adjoint_q1_2d_L6.npz")
    d = dict(np.load(fn))
    d["target"] = target
    save("ref_adjoint_q1_2d_L6", **d)
    # the reference's own matrices in its own numbering (2D Q1, levels 1..3) for the drop-in test
    R = po.run_ref(2, 1, 3, 1, rhs="sine", solver="pcg", nu=2, coarse="direct", tol=1e-8, dump_matrices=True)
    pre = R["prefix"]
    arrays = {"u_feat_order": np.fromfile(pre + ".u", dtype=np.float64), "iters": R["info"]["iters"],
              "rhs_feat_order": np.fromfile(pre + ".rhs", dtype=np.float64)}
    for l in (1, 2, 3):
        for mat in ("A", "P", "R"):
            if mat != "A" and l == 1:
                continue
            for part, dt in (("rowptr", np.uint64), ("col", np.uint64), ("val", np.float64)):
                arrays[f"L{l}_{mat}_{part}"] = np.fromfile(f"{pre}.L{l}.{mat}.{part}", dtype=dt)
        arrays[f"L{l}_filter"] = np.fromfile(f"{pre}.L{l}.filter", dtype=np.uint64)
        arrays[f"L{l}_lattice"] = np.fromfile(f"{pre}.L{l}.lattice", dtype=np.uint64)
    save("ref_matrices_q1_2d_L3", **arrays)
    cycles()
    feat_files()
    numbering()


if __name__ == "__main__":
    main()
