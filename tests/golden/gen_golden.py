"""Generate the golden fixtures of tests/golden/ from the REFERENCE's own solver.

Runs oracle/_ref/feat_ref (FEAT3's CPU multigrid, compiled from the reference sources by
oracle/Makefile; see oracle/ref_harness/feat_ref_driver.cpp) on small cases of every
configuration this project measures and stores its outputs, mapped to the lexicographic
lattice numbering through the DOF coordinates, as compressed .npz files:

    python tests/golden/gen_golden.py          # needs oracle/_ref/feat_ref
    python tests/golden/gen_golden.py --cycles # only the F/W-cycle and adaptive-CGC fixtures
    python tests/golden/gen_golden.py --files  # only the container-file fixtures (feat_files_q1_2d_L3/)
    python tests/golden/gen_golden.py --numbering  # only FEAT's DOF and cell numbering (ref_numbering.npz)
    python tests/golden/gen_golden.py --full [c2 c3 c4 c5]  # the measured configurations at full size (ref_c*_full_*)

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


def sampled(R, stride):
    """the reference's solution (and gradient) at every `stride`-th lattice DOF (element), plus
    norms of the whole vectors: the full-size vectors are too large to keep in the repository"""
    u = R["u"]
    out = {"u_stride": stride, "u_sample": u[::stride].copy(), "u_norm2": np.linalg.norm(u),
           "u_sum": u.sum(), "ndofs": u.size}
    if "grad" in R:
        out["grad_sample"] = R["grad"][::stride].copy()
        out["grad_norm2"] = np.linalg.norm(R["grad"])
    if "lambda" in R:
        out["lambda_sample"] = R["lambda"][::stride].copy()
        out["lambda_norm2"] = np.linalg.norm(R["lambda"])
    return out


def run_full(name, dim, degree, level, rhs, k=None, k_rule=None, stride=97, **kw):
    R = po.run_ref(dim, degree, level, 1, rhs=rhs, k=k, **kw)
    info = R["info"]
    arrays = dict(dim=dim, degree=degree, level=level, level_min=1, rhs_kind=rhs, iters=info["iters"],
                  status=info["status"], hist=info["hist"], solve_time=info["solve_time"],
                  setup_time=info["setup_time"], cfg=repr({k_: v for k_, v in kw.items() if k_ != "target"}),
                  **sampled(R, stride))
    if k is not None:
        arrays["k_rule"] = k_rule
        arrays["k_checksum"] = np.array([k.sum(), (k * k).sum()])
    save(name, **arrays)
    shutil.rmtree(R["workdir"], ignore_errors=True)
    return R


def lognormal(n, sigma, seed):
    return np.exp(sigma * np.random.default_rng(seed).standard_normal(n))


def full(which=("c2", "c3", "c4", "c5")):
    """The measured configurations at their full sizes, solved by the reference itself (minutes of
    CPU and up to ~30 GB of memory for the 257^3 case). Coefficient fields are regenerated from
    the stated rule (numpy default_rng(seed).standard_normal), and their checksums are stored."""
    pcg = dict(solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
    if "c2" in which:
        full_c2(pcg)
    if "c3" in which:
        full_c3(pcg)
    if "c4" in which:
        full_c4(pcg)
    if "c5" in which:
        full_c5(pcg)


def full_c2(pcg):
    # C2: 3D Q1, 65^3, f = 3 pi^2 prod sin(pi x_i); FP64 MG-PCG V(2,2), and the mixed form FP64
    # Richardson around ConvertPrecond(FP32 MG) (kernel/solver/convert_precond.hpp:41-120)
    run_full("ref_c2_full_q1_3d_L6", 3, 1, 6, "sine", **pcg)
    run_full("ref_c2_full_mixed_richardson_q1_3d_L6", 3, 1, 6, "sine",
             **dict(pcg, solver="richardson", inner="f32"))


def full_c3(pcg):
    # C3: 2D Q2, 1025^2, k = exp(N(0,1)) per element (seed 3), f = 1; FP64, and FP16-quantised inner matrices
    k3 = lognormal(512 * 512, 1.0, 3)
    run_full("ref_c3_full_q2_2d_L9", 2, 2, 9, "one", k=k3, k_rule="exp(default_rng(3).standard_normal(512^2))",
             **pcg)
    run_full("ref_c3_full_f16_q2_2d_L9", 2, 2, 9, "one", k=k3, k_rule="exp(default_rng(3).standard_normal(512^2))",
             **dict(pcg, inner="f16"))


def full_c4(pcg):
    # C4: adjoint on 2D Q1, 513^2, g ~ N(0, 0.25) (sigma 0.5, seed 21), u_target = u(k = 1) + N(0, 1e-2)
    # noise (sigma 1e-2, seed 22); the reference's FP64 adjoint (dJ/dk_e = -lambda_e^T K_e u_e)
    lvl = 9
    u1 = po.run_ref(2, 1, lvl, 1, rhs="one", solver="pcg", nu=2, omega_jac=0.5, coarse="direct", tol=1e-14)["u"]
    target = u1 + 1e-2 * np.random.default_rng(22).standard_normal(u1.size)
    k4 = lognormal(512 * 512, 0.5, 21)
    R = run_full("ref_c4_full_adjoint_q1_2d_L9", 2, 1, lvl, "one", k=k4,
                 k_rule="exp(0.5 * default_rng(21).standard_normal(512^2))", target=target, stride=7,
                 **dict(pcg, tol=1e-14))
    fn = os.path.join(HERE, "ref_c4_full_adjoint_q1_2d_L9.npz")
    d = dict(np.load(fn))
    d["target_rule"] = "u(k=1, tol 1e-14) + 1e-2 * default_rng(22).standard_normal(513^2)"
    d["target_checksum"] = np.array([target.sum(), (target * target).sum()])
    d["J"] = 0.5 * float(np.sum((R["u"] - target) ** 2))
    save("ref_c4_full_adjoint_q1_2d_L9", **d)


def full_c5(pcg):
    # C5: 3D Q1, 257^3, k = exp(N(0,1)) per element (seed 2026: the benchmark's field), f = 1
    k5 = lognormal(256 ** 3, 1.0, 2026)
    run_full("ref_c5_full_q1_3d_L8", 3, 1, 8, "one", k=k5, k_rule="exp(default_rng(2026).standard_normal(256^3))",
             stride=997, **pcg)


def main():
    if not po.have_ref():
        sys.exit("oracle/_ref/feat_ref is missing: build it with `make -C oracle ref` first")
    if "--full" in sys.argv:
        sel = [a for a in sys.argv[1:] if a in ("c2", "c3", "c4", "c5")]
        return full(sel or ("c2", "c3", "c4", "c5"))
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
