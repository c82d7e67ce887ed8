"""The per-element OP2 user kernels of include/ins_solver_b200/op2_kernels.h
against the reference's own kernels (src/kernels/*.h, compiled into
oracle/_ref by oracle/Makefile): every kernel the header provides has the
reference's name and argument list (types and names) and gives the
reference's values on the same random cell / face data, for 2D and 3D at
p = 1..4."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import oracle_py as O
import sipg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ins_solver_b200", "op2_kernels.h")
LIB_SRC = os.path.join(ROOT, "tests", "cpp", "op2_kernels_lib.cpp")
REF_GEN = os.path.join(ROOT, "oracle", "_ref", "gen")

# kernels on a pair of cells sharing a face (faceNum = {face in L, face in R})
PAIR = {"fvmf_3d_calc_tau_faces", "fvmf_2d_calc_tau_faces", "vmf_calc_tau_faces", "fvmf_3d_op2_diag",
        "fvmf_2d_op2_diag", "fvmf_3d_op2_block_diag", "fvmf_2d_op2_block_diag"}
# kernels on one boundary face of a cell
BFACE = {"fvmf_3d_calc_tau_bfaces", "fvmf_2d_calc_tau_bfaces", "vmf_calc_tau_bfaces", "vmf_3d_mult_avg_jump",
         "vmf_2d_mult_avg_jump", "fvmf_3d_apply_bc", "fvmf_2d_apply_bc", "vmf_3d_apply_bc", "vmf_2d_apply_bc",
         "fvmf_3d_bop_diag", "fvmf_2d_bop_diag", "fvmf_3d_bop_block_diag", "fvmf_2d_bop_block_diag"}
SCALARS = {"alpha", "beta", "residual", "tmp_alpha_0", "tmp_alpha_1", "constant", "mmConst"}
MATS = {"u_pre_mat", "v_pre_mat", "w_pre_mat", "op1", "op1L", "op1R"}
# kernels every (shared) build has; the others belong to the dimension in their name
SHARED = {"constant_mult", "copy_dg_np", "copy_dg_np_mat", "reciprocal", "zero_npf_3", "poisson_pr_fact",
          "poisson_vis_fact", "vmf_calc_tau_faces", "vmf_calc_tau_bfaces"}


def split_args(s):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
            continue
        depth += {"(": 1, ")": -1}.get(ch, 0)
        cur += ch
    out.append(cur)
    res = []
    for a in out:
        a = " ".join(a.split())
        m = re.match(r"^(.*?)(\w+)$", a)
        res.append((m.group(1).replace(" *", "*").replace("* ", "*").strip(), m.group(2)))
    return res


def header_kernels():
    """name -> (template parameters, [(type, name)]) of the header's kernels."""
    text = open(HEADER).read()
    while "namespace detail {" in text:  # helpers are not kernels
        a = text.index("namespace detail {")
        text = text[:a] + text[text.index("}  // namespace detail", a) + 1:]
    out = {}
    for m in re.finditer(r"template <([^>]*)>\s*SIPG_OP2_HD void (\w+)\(([^)]*)\)", text):
        out[m.group(2)] = (m.group(1).strip(), split_args(m.group(3)))
    return out


def ref_signature(dim, order, name):
    path = os.path.join(REF_GEN, f"d{dim}p{order}", name + ".h")
    text = open(path).read()
    m = re.search(r"inline void (\w+)\(([^)]*)\)", text)
    return split_args(m.group(2))


def kernel_dim(name):
    if name in SHARED:
        return None
    return 3 if name.startswith(("fvmf_3d", "vmf_3d", "cg3_")) else 2


def ref_names(dim):
    with open(os.path.join(REF_GEN, f"d{dim}p1", "all.h")) as f:
        return [l.split('"')[1][:-2] for l in f if l.startswith("#include")]


@pytest.fixture(scope="module")
def libs(tmp_path_factory):
    if not O.have_ref():
        pytest.skip("oracle/_ref not built (the reference tree is not available)")
    ours = header_kernels()
    d = tmp_path_factory.mktemp("op2")
    lines = []
    for dim in (2, 3):
        for p in (1, 2, 3, 4):
            lines.append(f"template <> int call_kernel<{dim}, {p}>(const char* name, void** a) {{")
            for name, (tpl, args) in ours.items():
                if kernel_dim(name) not in (None, dim):
                    continue
                targs = f"<{p}>" if tpl == "int ORDER" else f"<{dim}, {p}>"
                casts = ", ".join(f"({t})a[{i}]" for i, (t, _) in enumerate(args))
                lines.append(f'  if (!std::strcmp(name, "{name}")) {{ op2::{name}{targs}({casts}); return 0; }}')
            lines.append("  return -1;\n}")
    (d / "op2_dispatch.inc").write_text("\n".join(lines) + "\n")
    so = d / "libop2k.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{d}", LIB_SRC, "-o", str(so)], check=True)
    mine = C.CDLL(str(so))
    mine.op2_kernel.restype = C.c_int
    ref = O.ref_lib()
    ref.ref_kernel.restype = C.c_int
    return ours, mine, ref


def table_mesh(dim, order):
    t = sipg.ref_tables(dim, order)
    e = {"K": 0, "F": 0, "Kb": 0}
    for k in ("geof", "nx", "ny", "nz", "sJ", "fscale"):
        e[k] = np.zeros(1)
    for k in ("face2cells", "faceNum", "fmaskL", "fmaskR", "bface2cell", "bfaceNum"):
        e[k] = np.zeros(1, np.int32)
    return t, O.OMesh(t, e)


def make_args(name, args, t, rng):
    """One random set of arguments; returns (list of numpy objects or lists, outputs to compare)."""
    dim, Np, Nfp, Nf = t["dim"], t["Np"], t["Nfp"], t["Nf"]
    ng = 10 if dim == 3 else 5
    fL, fR = int(rng.integers(Nf)), int(rng.integers(Nf))
    vals = []
    for typ, an in args:
        const = typ.startswith("const")
        if typ.endswith("**"):
            n = {"factor": Np, "tau": Nf, "geof": ng}[an]
            vals.append(("pp", [rng.uniform(0.5, 1.5, n) for _ in range(2)], const))
        elif "int" in typ:
            if an == "faceNum":
                v = [fL, fR] if name in PAIR else [fL]
            elif an.endswith("bc_type"):
                v = [int(rng.integers(3))]
            elif an in ("fmaskR_corrected", "fmaskL_corrected"):
                v = list(t["fmask"][fR if an == "fmaskR_corrected" else fL])
                if rng.integers(2):
                    v = v[::-1]
            else:
                raise AssertionError(f"no rule for int argument {an} of {name}")
            vals.append(("i", np.array(v, np.int32), const))
        elif "bool" in typ:
            vals.append(("b", np.array([bool(rng.integers(2))]), const))
        else:
            if an in SCALARS or (an == "mm_factor" and name.startswith("vmf_")):
                n = 1
            elif an == "geof":
                n = ng
            elif an in ("nx", "ny", "nz", "sJ", "fscale"):
                n = 2 if name in PAIR else 1 if name in BFACE else Nf
            elif an == "tau":
                n = Nf
            elif "jump" in an or "avg" in an or (name == "zero_npf_3"):
                n = Nf * Nfp
            elif an in MATS or name == "copy_dg_np_mat":
                n = Np * Np
            else:
                n = Np
            lo = -1.0 if an in ("nx", "ny", "nz") else 0.5
            vals.append(("d", rng.uniform(lo, 1.5, n), const))
    return vals


def pointers(vals):
    keep, ptrs = [], []
    for kind, v, _ in vals:
        if kind == "pp":
            arrs = [np.array(a) for a in v]
            pp = (C.POINTER(C.c_double) * 2)(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
            keep.append((arrs, pp))
            ptrs.append(C.cast(pp, C.c_void_p))
        else:
            a = np.array(v)
            keep.append(a)
            ptrs.append(a.ctypes.data_as(C.c_void_p))
    return keep, (C.c_void_p * len(ptrs))(*ptrs)


def test_every_provided_kernel_has_the_reference_argument_list(libs):
    ours, _, _ = libs
    checked = 0
    for dim in (2, 3):
        for name in ref_names(dim):
            if name not in ours:
                continue
            assert ours[name][1] == ref_signature(dim, 3, name), name
            checked += 1
    assert checked >= 60


@pytest.mark.parametrize("dim,order", [(2, 1), (2, 2), (2, 3), (2, 4), (3, 1), (3, 2), (3, 3), (3, 4)])
def test_kernels_match_the_reference_kernels(libs, dim, order):
    ours, mine, ref = libs
    t, om = table_mesh(dim, order)
    rng = np.random.default_rng(100 * dim + order)
    names = [n for n in ref_names(dim) if n in ours]
    assert len(names) >= 30
    for name in names:
        for trial in range(6):
            vals = make_args(name, ours[name][1], t, rng)
            ka, pa = pointers(vals)
            kb, pb = pointers(vals)
            assert mine.op2_kernel(C.byref(om.s), name.encode(), pa) == 0, name
            assert ref.ref_kernel(C.byref(om.s), name.encode(), pb) == 0, name
            for (kind, _, const), a, b in zip(vals, ka, kb):
                if const:
                    continue
                xa = a[0] if kind == "pp" else [a]
                xb = b[0] if kind == "pp" else [b]
                for u, v in zip(xa, xb):
                    scale = max(1.0, float(np.abs(v).max()))
                    assert np.abs(u - v).max() <= 1e-13 * scale, (name, trial)
