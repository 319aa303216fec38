"""H_eff * psi and Lanczos on the GPU against the reference (golden) and the oracle.

Tolerances: FP64 path 1e-12 of max|H psi| (sum order differs from the
reference's BLAS); 3xTF32 path 2e-6 of max|H psi| (split TF32 products, FP32
partial sums per task term); Lanczos energies 1e-10 relative.
"""
import numpy as np
import pytest

from conftest import centre_files, fixture_tensor, tensor_names
from oracle.blocks import from_npz, parse_meta
from oracle.heff import heff_apply

pytestmark = pytest.mark.gpu


def build_problem(path):
    import sadmrg
    z = np.load(path)
    m = parse_meta(z)
    names = tensor_names(z)
    h = sadmrg.Handle(sym=m["sym"], cplx=bool(m["cplx"]))
    psi = fixture_tensor(z, "psi")
    hl = fixture_tensor(z, "hh_il") if "hh_il" in names else None
    hr = fixture_tensor(z, "hh_ir") if "hh_ir" in names else None
    il, ir, ns = m["il"], m["ir"], m["ns"]
    # the reference's operator set (src/dmrg_inst.cpp:309-351), right operators summed with couplings
    ops, terms = [], []
    oprl = {int(n.split("_")[-1]): n for n in names if n.startswith("opr_il_")}
    oprr = {int(n.split("_")[-1]): n for n in names if n.startswith("opr_ir_")}
    if il < ns // 2:
        m1, m4 = il + 1, ns - ir
    else:
        m1, m4 = ns - ir, il + 1
    sym = m["sym"]
    for m0 in range(m1):
        acc = None
        for mm in range(m4):
            j, k = (m0, ir + mm) if il < ns // 2 else (mm, ir + m0)
            hv = m["hmap"].get((j, k), 0)
            src = (oprr.get(k) if il < ns // 2 else oprl.get(j))
            if hv > 0 and src is not None:
                t = from_npz(z, src, sym)
                if acc is None:
                    acc = t
                    acc.blocks = {kk: m["coup"][hv] * v for kk, v in t.blocks.items()}
                else:
                    for kk, v in t.blocks.items():
                        acc.blocks[kk] = acc.blocks.get(kk, 0) + m["coup"][hv] * v
        if acc is None:
            continue
        fixed = oprl.get(m0) if il < ns // 2 else oprr.get(ir + m0)
        if fixed is None:
            continue
        keys = sorted(acc.blocks, key=acc.index)
        summed = sadmrg.BlockTensorData(acc.dirs, [b[0] for b in acc.bonds], [b[1] for b in acc.bonds],
                                        acc.locspin, np.array([acc.index(k) for k in keys], np.int64),
                                        np.concatenate([acc.blocks[k].reshape(-1, order="F") for k in keys]))
        ops.append(fixture_tensor(z, fixed))
        ops.append(summed)
        a, b = len(ops) - 2, len(ops) - 1
        terms.append((a, b) if il < ns // 2 else (b, a))
    h.heff_plan(psi, hl, hr, ops, terms)
    return h, z, m, psi


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_heff_fp64_matches_reference(path):
    import sadmrg
    h, z, m, psi = build_problem(path)
    ref = np.array(z["hpsi__data"])
    out = h.heff_apply(psi.data, sadmrg.PREC_FP64)
    assert out.shape == ref.shape
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    info = h.heff_info()
    assert info["flops"] > 0 and info["n"] == ref.size


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_heff_tf32x3_close_to_fp64(path):
    import sadmrg
    h, z, m, psi = build_problem(path)
    ref = np.array(z["hpsi__data"])
    out = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
    np.testing.assert_allclose(out, ref, rtol=0, atol=2e-6 * np.abs(ref).max())


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_heff_random_vectors_match_oracle(path):
    """linearity + oracle on seeded random psi of the same structure"""
    import sadmrg
    h, z, m, psi = build_problem(path)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(psi.data.shape)
    if np.iscomplexobj(psi.data):
        x = x + 1j * rng.standard_normal(psi.data.shape)
    y = h.heff_apply(x, sadmrg.PREC_FP64)
    # oracle on the same vector
    sym = m["sym"]
    names = tensor_names(z)
    opsi = from_npz(z, "psi", sym)
    keys = sorted(opsi.blocks, key=opsi.index)
    off = 0
    for k in keys:
        n = opsi.blocks[k].size
        opsi.blocks[k] = x[off:off + n].reshape(opsi.blocks[k].shape, order="F")
        off += n
    hl = from_npz(z, "hh_il", sym) if "hh_il" in names else None
    hr = from_npz(z, "hh_ir", sym) if "hh_ir" in names else None
    ol = {int(n.split("_")[-1]): from_npz(z, n, sym) for n in names if n.startswith("opr_il_")}
    orr = {int(n.split("_")[-1]): from_npz(z, n, sym) for n in names if n.startswith("opr_ir_")}
    ref = heff_apply(opsi, hl, hr, ol, orr, m["hmap"], m["coup"], m["il"], m["ir"], m["ns"]).flat()
    np.testing.assert_allclose(y, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    y2 = h.heff_apply(2.0 * x, sadmrg.PREC_FP64)
    np.testing.assert_allclose(y2, 2.0 * y, rtol=0, atol=1e-13 * np.abs(y).max())


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_lanczos_energy_matches_reference(path):
    import sadmrg
    h, z, m, psi = build_problem(path)
    n = psi.data.size
    mlanc = min(40, n + 1)
    e, v, mv = h.heff_lanczos(psi.data, mlanc, sadmrg.PREC_FP64)
    assert abs(e - m["lanczos_E"]) <= 1e-10 * abs(m["lanczos_E"])
    # Ritz vector is normalised and an eigenvector to the Lanczos tolerance
    assert abs(np.vdot(v, v).real - 1.0) < 1e-12
    hv = h.heff_apply(v, sadmrg.PREC_FP64)
    assert np.linalg.norm(hv - e * v) < 1e-4 * abs(e)
    em, vm, mvm = h.heff_lanczos(psi.data, mlanc, sadmrg.PREC_TF32X3)
    assert abs(em - m["lanczos_E"]) <= 1e-10 * abs(m["lanczos_E"])
