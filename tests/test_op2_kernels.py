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
PAIR = {"ins_proj_setup_0", "fvmf_3d_calc_tau_faces", "fvmf_2d_calc_tau_faces", "vmf_calc_tau_faces", "fvmf_3d_op2_diag",
        "fvmf_2d_op2_diag", "fvmf_3d_op2_block_diag", "fvmf_2d_op2_block_diag"}
# kernels on one boundary face of a cell
BFACE = {"fvmf_3d_calc_tau_bfaces", "fvmf_2d_calc_tau_bfaces", "vmf_calc_tau_bfaces", "vmf_3d_mult_avg_jump",
         "vmf_2d_mult_avg_jump", "fvmf_3d_apply_bc", "fvmf_2d_apply_bc", "vmf_3d_apply_bc", "vmf_2d_apply_bc",
         "fvmf_3d_bop_diag", "fvmf_2d_bop_diag", "fvmf_3d_bop_block_diag", "fvmf_2d_bop_block_diag"}
SCALARS = {"alpha", "beta", "residual", "tmp_alpha_0", "tmp_alpha_1", "constant", "mmConst", "dt", "a0", "a1", "h",
           "pen", "pen_f", "iter_g", "b0", "b1", "_div_factor", "fact0", "fact1", "art_vis"}
# per cell face-node data (DG_NUM_FACES x DG_NPF)
FACE_DATS = {"dPdN", "dPdN_old", "dPdNOld"}
# kernels whose `factor` is a scalar
SCALAR_FACTOR = {"ins_3d_proj_pen", "ins_2d_proj_pen"}
MATS = {"u_pre_mat", "v_pre_mat", "w_pre_mat", "op1", "op1L", "op1R"}
# kernels every (shared) build has; the others belong to the dimension in their name
SHARED = {"constant_mult", "copy_dg_np", "copy_dg_np_mat", "reciprocal", "zero_npf_3", "poisson_pr_fact",
          "poisson_vis_fact", "vmf_calc_tau_faces", "vmf_calc_tau_bfaces", "ins_proj_setup_0", "ins_proj_setup_1",
          "mp_ins_pr_bc_dpdn_factors", "mp_ins_pr_div_factor"}
# kernels provided per build (the shared ones in both)
PER_BUILD = {2: 48, 3: 50}


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
    return 3 if name.startswith(("fvmf_3d", "vmf_3d", "cg3_", "ins_3d_", "mp_ins_3d_")) else 2


def ref_names(dim):
    with open(os.path.join(REF_GEN, f"d{dim}p1", "all.h")) as f:
        return [l.split('"')[1][:-2] for l in f if l.startswith("#include")]


def build_lib(d, ours, defines=()):
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
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{d}", *defines, LIB_SRC, "-o", str(so)],
                   check=True)
    lib = C.CDLL(str(so))
    lib.op2_kernel.restype = C.c_int
    return lib


@pytest.fixture(scope="module")
def libs(tmp_path_factory):
    if not O.have_ref():
        pytest.skip("oracle/_ref not built (the reference tree is not available)")
    ours = header_kernels()
    mine = build_lib(tmp_path_factory.mktemp("op2"), ours)
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


def make_args(name, args, t, rng, bc_mode=None):
    """One random set of arguments: (kind, values, const) per argument. bc_mode
    0 / 1 / 2 gives every component that boundary type, None random types."""
    dim, Np, Nfp, Nf = t["dim"], t["Np"], t["Nfp"], t["Nf"]
    ng = 10 if dim == 3 else 5
    fL, fR = int(rng.integers(Nf)), int(rng.integers(Nf))
    vals = []
    for typ, an in args:
        const = typ.startswith("const")
        if typ.endswith("**"):
            n = {"factor": Np, "tau": Nf, "geof": ng, "f0": Nf * Nfp}[an]
            vals.append(("pp", [rng.uniform(0.5, 1.5, n) for _ in range(2)], const))
        elif "int" in typ:
            if an == "faceNum":
                v = [fL, fR] if name in PAIR else [fL]
            elif an.endswith("bc_type"):
                v = [int(rng.integers(3)) if bc_mode is None else bc_mode]
            elif an in ("cell_g", "conv_g"):
                v = [int(rng.integers(5))]
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
            if an in SCALARS or (an == "mm_factor" and name.startswith("vmf_")) or \
                    (an == "factor" and name in SCALAR_FACTOR):
                n = 1
            elif an == "geof":
                n = ng
            elif an in ("nx", "ny", "nz", "sJ", "fscale"):
                n = 2 if name in PAIR else 1 if name in BFACE else Nf
            elif an == "tau":
                n = Nf
            elif "jump" in an or "avg" in an or (name == "zero_npf_3") or an in FACE_DATS:
                n = Nf * Nfp
            elif an.endswith("_bc"):
                n = Nfp
            elif an in MATS or an.endswith("_op1") or name == "copy_dg_np_mat":
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
    assert checked == PER_BUILD[2] + PER_BUILD[3]  # the shared ones counted in both builds


@pytest.mark.parametrize("dim,order", [(2, 1), (2, 2), (2, 3), (2, 4), (3, 1), (3, 2), (3, 3), (3, 4)])
def test_kernels_match_the_reference_kernels(libs, dim, order):
    ours, mine, ref = libs
    t, om = table_mesh(dim, order)
    rng = np.random.default_rng(100 * dim + order)
    names = [n for n in ref_names(dim) if n in ours]
    assert len(names) == PER_BUILD[dim]
    for name in names:
        for trial in range(6):
            # Dirichlet, Neumann and slip on every component, then random mixes
            vals = make_args(name, ours[name][1], t, rng, bc_mode=trial if trial < 3 else None)
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


def test_corrected_forms_without_the_reference_quirks(tmp_path):
    """SIPG_OP2_REF_QUIRKS=0: the volume block is J sum_d D_d^T M F D_d and the
    constant-coefficient flux keeps the n_z term of n . {grad u}."""
    ours = header_kernels()
    lib = build_lib(tmp_path, ours, ("-DSIPG_OP2_REF_QUIRKS=0",))
    rng = np.random.default_rng(5)
    for dim, order in ((2, 3), (3, 2)):
        t, om = table_mesh(dim, order)
        Np, Nfp, Nf = t["Np"], t["Nfp"], t["Nf"]
        geof = rng.uniform(0.5, 1.5, 10 if dim == 3 else 5)
        f = rng.uniform(0.5, 1.5, Np)
        op1 = np.zeros(Np * Np)
        keep, args = pointers([("d", geof, True), ("d", f, True), ("d", op1, False)])
        assert lib.op2_kernel(C.byref(om.s), f"fvmf_{dim}d_op1".encode(), args) == 0
        G = geof[:dim * dim].reshape(dim, dim)
        Dref = [t["Dr"], t["Ds"], t["Dt"]][:dim]
        want = np.zeros((Np, Np))
        for d in range(dim):
            Dd = sum(G[r, d] * Dref[r] for r in range(dim))
            want += Dd.T @ t["M"] @ np.diag(f) @ Dd
        want *= geof[dim * dim]
        got = keep[2].reshape(Np, Np).T  # column-major
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    t, om = table_mesh(3, 2)
    Nf, Nfp = t["Nf"], t["Nfp"]
    n = [rng.uniform(-1, 1, Nf) for _ in range(3)]
    sJ, tau = rng.uniform(0.5, 1.5, Nf), rng.uniform(0.5, 1.5, Nf)
    jump = rng.uniform(-1, 1, Nf * Nfp)
    avg = [rng.uniform(-1, 1, Nf * Nfp) for _ in range(3)]
    bufs = [("d", n[0], True), ("d", n[1], True), ("d", n[2], True), ("d", sJ, True), ("d", tau, True)]
    for c in range(3):
        bufs += [("d", jump.copy(), False)] + [("d", a.copy(), False) for a in avg]
    keep, args = pointers(bufs)
    assert lib.op2_kernel(C.byref(om.s), b"vmf_3d_mult_flux", args) == 0
    fi = np.repeat(np.arange(Nf), Nfp)
    s_full = n[0][fi] * avg[0] + n[1][fi] * avg[1] + n[2][fi] * avg[2]
    want = sJ[fi] * (tau[fi] * 0.5 * jump - s_full)
    assert np.abs(keep[5] - want).max() <= 1e-13


def test_kernels_compile_into_a_device_kernel(tmp_path):
    """The header's kernels are __host__ __device__: a CUDA kernel that calls them
    (per element, tables in device memory) compiles for sm_100a."""
    src = tmp_path / "op2_device.cu"
    src.write_text(f"""
#include "{HEADER}"
namespace op2 = ins_solver_b200::op2;
__device__ op2::RefTables g_tables;
namespace ins_solver_b200 {{ namespace op2 {{
template <> __host__ __device__ const RefTables& ref_tables<3, 3>() {{
#ifdef __CUDA_ARCH__
  return g_tables;
#else
  static RefTables h{{}};
  return h;
#endif
}}
}} }}
__global__ void cells(const double* geof, const double* f, double* op1, double* diag, double* r, const double* Ap,
                      double* res, int* counts, double* iters) {{
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  op2::fvmf_3d_op1<3>(geof + 10 * e, f + 20 * e, op1 + 400 * e);
  op2::fvmf_3d_op1_diag<3>(geof + 10 * e, f + 20 * e, diag + 20 * e);
  const double alpha = 0.5;
  op2::cg3_update_res<3>(&alpha, res + e, Ap + 60 * e, Ap + 60 * e + 20, Ap + 60 * e + 40, r + 60 * e,
                         r + 60 * e + 20, r + 60 * e + 40);
  op2::ins_3d_proj_cg_precon<3>(geof + 10 * e, res + e, Ap + 60 * e, Ap + 60 * e + 20, Ap + 60 * e + 40,
                                r + 60 * e, r + 60 * e + 20, r + 60 * e + 40, counts, counts + 1, iters);
}}
""")
    out = tmp_path / "op2_device.o"
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-c", str(src), "-o",
                    str(out)], check=True)
    assert out.stat().st_size > 0
