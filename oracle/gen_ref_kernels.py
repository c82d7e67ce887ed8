#!/usr/bin/env python3
"""Specialise the reference's OP2 user kernels for the CPU reference build.

TEST INFRASTRUCTURE ONLY: part of the recipe that compiles the reference's own
kernel sources (src/kernels/*.h of TobyFlynn/INS-Solver) into oracle/_ref/.

The reference ships its kernels as order-generic headers that its build turns
into plain C++ by textual substitution (DG_FP, DG_NP, DG_NPF, DG_NUM_FACES,
DG_ORDER) and by expanding op2_in_kernel_gemv / op2_in_kernel_gemm into loops
(the OP2_DG_CUDA branch of its code generator). This script performs those same
substitutions, with its own code, for one (dimension, order) at a time and
writes the specialised headers to oracle/_ref/gen/d<dim>p<order>/. Nothing is
written under the reference tree.

usage: gen_ref_kernels.py <reference_root> <out_dir>
"""
import os
import sys

KERNELS_3D = [
    "fvmf_3d_grad", "fvmf_3d_calc_tau_faces", "fvmf_3d_calc_tau_bfaces", "vmf_3d_mult_avg_jump",
    "fvmf_3d_mult_flux", "vmf_3d_mult_flux", "vmf_3d_mult_cells_geof", "fvmf_3d_mult_mm_geof",
    "fvmf_3d_apply_bc", "fvmf_3d_op1_diag", "fvmf_3d_op2_diag", "fvmf_3d_mm_diag",
    "fvmf_3d_bop_diag", "fvmf_3d_op1", "fvmf_3d_op2_block_diag", "fvmf_3d_mm_block_diag",
    "fvmf_3d_bop_block_diag", "vmf_calc_tau_faces", "vmf_calc_tau_bfaces",
    "cg3_alpha", "cg3_alpha_pre", "cg3_compute_beta", "cg3_compute_beta_pre",
    "cg3_compute_beta_pre_flex", "cg3_update_ans", "cg3_update_res", "cg3_update_p",
    "cg3_residual", "cg3_jacobi", "cg3_block_jacobi", "zero_npf_3", "copy_dg_np",
    "cg3_recp_factor_inv_mass", "vmf_3d_mult_mm_geof", "vmf_3d_apply_bc",
    "constant_mult", "reciprocal", "copy_dg_np_mat", "poisson_pr_fact", "poisson_vis_fact",
    "ins_3d_proj_rhs", "ins_3d_proj_pen", "ins_3d_proj_cg_precon", "ins_proj_setup_0", "ins_proj_setup_1",
    "ins_3d_pr_1", "mp_ins_3d_pr_2", "mp_ins_pr_bc_dpdn_factors", "mp_ins_pr_div_factor", "mp_ins_3d_vis_0",
    "ins_3d_advec_0", "ins_3d_advec_1", "ins_3d_advec_2", "ins_3d_advec_3", "mp_ins_3d_pr_mu", "mp_ins_3d_pr_0",
    "advec_3d_0", "advec_3d_flux", "ls_advec_3d_bc", "runge_kutta_0", "runge_kutta_1", "ls_step",
]
KERNELS_2D = [
    "fvmf_2d_grad", "fvmf_2d_calc_tau_faces", "fvmf_2d_calc_tau_bfaces", "vmf_2d_mult_avg_jump",
    "fvmf_2d_mult_flux", "vmf_2d_mult_cells_geof", "fvmf_2d_mult_mm_geof", "fvmf_2d_apply_bc",
    "fvmf_2d_op1_diag", "fvmf_2d_op2_diag", "fvmf_2d_mm_diag", "fvmf_2d_bop_diag",
    "fvmf_2d_op1", "fvmf_2d_op2_block_diag", "fvmf_2d_mm_block_diag", "fvmf_2d_bop_block_diag",
    "vmf_calc_tau_faces", "vmf_calc_tau_bfaces",
    "cg_alpha", "cg_alpha_pre", "cg_compute_beta", "cg_compute_beta_pre",
    "cg_compute_beta_pre_flex", "cg_update_ans", "cg_update_res", "cg_update_p",
    "cg_residual", "cg_jacobi", "cg_block_jacobi", "zero_npf_3", "copy_dg_np",
    "cg_recp_factor_inv_mass", "vmf_2d_mult_flux", "vmf_2d_mult_mm_geof", "vmf_2d_apply_bc",
    "constant_mult", "reciprocal", "copy_dg_np_mat", "poisson_pr_fact", "poisson_vis_fact",
    "ins_2d_proj_rhs", "ins_2d_proj_pen", "ins_proj_cg_2d", "ins_proj_setup_0", "ins_proj_setup_1",
    "ins_pressure_rhs_2d", "mp_ins_pr_bc_dpdn_factors", "mp_ins_pr_div_factor",
]


def np_of(dim, p):
    return (p + 1) * (p + 2) // 2 if dim == 2 else (p + 1) * (p + 2) * (p + 3) // 6


def nfp_of(dim, p):
    return p + 1 if dim == 2 else (p + 1) * (p + 2) // 2


def split_call(src, name):
    """Yield (start, end, args) for each `name(...)` call; end is past the ';'."""
    pos = 0
    while True:
        i = src.find(name + "(", pos)
        if i < 0:
            return
        j = i + len(name) + 1
        depth, k, args, cur = 1, j, [], ""
        while depth:
            ch = src[k]
            if ch == "(":
                depth += 1
            elif ch == ")":
                depth -= 1
                if depth == 0:
                    break
            if ch == "," and depth == 1:
                args.append(cur.strip())
                cur = ""
            else:
                cur += ch
            k += 1
        args.append(cur.strip())
        end = src.find(";", k) + 1
        yield i, end, args
        pos = end


def expand_gemv(src):
    """op2_in_kernel_gemv(trans, m, n, alpha, A, lda, x, beta, y) -> loops."""
    out, last = [], 0
    for s, e, a in list(split_call(src, "op2_in_kernel_gemv")):
        trans, m, n, alpha, A, _lda, x, beta, y = a
        t = "true" in trans
        outer, inner = (n, m) if t else (m, n)
        ind = "DG_MAT_IND(j, i, {m}, {n})" if t else "DG_MAT_IND(i, j, {m}, {n})"
        ind = ind.format(m=m, n=n)
        upd = (f"{y}[i] = ({alpha}) * tmp_gemv;" if beta.strip() == "0.0"
               else f"{y}[i] = ({beta}) * {y}[i] + ({alpha}) * tmp_gemv;")
        code = (f"for(int i = 0; i < {outer}; i++) {{\n  double tmp_gemv = 0.0;\n"
                f"  for(int j = 0; j < {inner}; j++) {{\n    int ind = {ind};\n"
                f"    tmp_gemv += {A}[ind] * {x}[j];\n  }}\n  {upd}\n}}")
        out.append(src[last:s])
        out.append(code)
        last = e
    out.append(src[last:])
    return "".join(out)


def expand_gemm(src):
    """op2_in_kernel_gemm(tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc) -> loops."""
    out, last = [], 0
    for s, e, a in list(split_call(src, "op2_in_kernel_gemm")):
        tA, tB, m, n, k, alpha, A, _lda, B, _ldb, beta, C, _ldc = a
        ia = "DG_MAT_IND(k, i, {m}, {k})" if "true" in tA else "DG_MAT_IND(i, k, {m}, {k})"
        ib = "DG_MAT_IND(j, k, {k}, {n})" if "true" in tB else "DG_MAT_IND(k, j, {k}, {n})"
        ia, ib = ia.format(m=m, k=k), ib.format(k=k, n=n)
        upd = (f"{C}[c_ind] = ({alpha}) * tmp_gemm;" if beta.strip() == "0.0"
               else f"{C}[c_ind] = ({beta}) * {C}[c_ind] + ({alpha}) * tmp_gemm;")
        code = (f"for(int i = 0; i < {m}; i++) {{\n  for(int j = 0; j < {n}; j++) {{\n"
                f"    double tmp_gemm = 0.0;\n    for(int k = 0; k < {k}; k++) {{\n"
                f"      int a_ind = {ia};\n      int b_ind = {ib};\n"
                f"      tmp_gemm += {A}[a_ind] * {B}[b_ind];\n    }}\n"
                f"    int c_ind = DG_MAT_IND(i, j, {m}, {n});\n    {upd}\n  }}\n}}")
        out.append(src[last:s])
        out.append(code)
        last = e
    out.append(src[last:])
    return "".join(out)


def specialise(text, dim, p):
    text = expand_gemv(text)
    text = expand_gemm(text)
    text = text.replace("DG_FP", "double")
    text = text.replace("DG_NPF", str(nfp_of(dim, p)))
    text = text.replace("DG_NP", str(np_of(dim, p)))
    text = text.replace("DG_NUM_FACES", str(dim + 1))
    text = text.replace("DG_ORDER", str(p))
    return text


def signature(text):
    """(name, [arg type, ...]) of the first `inline void name(...)` in text."""
    i = text.index("inline void ")
    j = text.index("(", i)
    name = text[i + len("inline void "):j].strip()
    depth, k = 1, j + 1
    while depth:
        depth += {"(": 1, ")": -1}.get(text[k], 0)
        k += 1
    types = []
    for a in text[j + 1:k - 1].split(","):
        a = " ".join(a.split())
        cut = len(a)
        while cut > 0 and (a[cut - 1].isalnum() or a[cut - 1] == "_"):
            cut -= 1
        types.append(a[:cut].strip())
    return name, types


def dispatch(sigs):
    """Body of call_kernel(name, args): one branch per kernel, arguments cast from void*."""
    lines = ["static int call_kernel(const char *name, void **a) {"]
    for name, types in sigs:
        args = ", ".join(f"({t})a[{i}]" for i, t in enumerate(types))
        lines.append(f'  if (!std::strcmp(name, "{name}")) {{ {name}({args}); return 0; }}')
    lines.append("  return -1;\n}")
    return "\n".join(lines) + "\n"


def main():
    ref_root, out_dir = sys.argv[1], sys.argv[2]
    kdir = os.path.join(ref_root, "src", "kernels")
    for dim, names in ((2, KERNELS_2D), (3, KERNELS_3D)):
        for p in range(1, 5):
            d = os.path.join(out_dir, f"d{dim}p{p}")
            os.makedirs(d, exist_ok=True)
            sigs = []
            for n in names:
                with open(os.path.join(kdir, n + ".h")) as f:
                    text = f.read()
                spec = specialise(text, dim, p)
                sigs.append(signature(spec))
                with open(os.path.join(d, n + ".h"), "w") as f:
                    f.write(spec + "\n")
            with open(os.path.join(d, "all.h"), "w") as f:
                f.write("".join(f'#include "{n}.h"\n' for n in names))
            with open(os.path.join(d, "dispatch.inc"), "w") as f:
                f.write(dispatch(sigs))


if __name__ == "__main__":
    main()
