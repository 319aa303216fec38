"""The numpy oracle against the reference's own outputs (golden fixtures)."""
import numpy as np
import pytest

from conftest import centre_files, tensor_names
from oracle.blocks import from_npz, parse_meta
from oracle.heff import heff_apply
from oracle import cgc


def _load_heff_case(path):
    z = np.load(path)
    m = parse_meta(z)
    sym = m["sym"]
    names = tensor_names(z)
    psi = from_npz(z, "psi", sym)
    hl = from_npz(z, "hh_il", sym) if "hh_il" in names else None
    hr = from_npz(z, "hh_ir", sym) if "hh_ir" in names else None
    ol = {int(n.split("_")[-1]): from_npz(z, n, sym) for n in names if n.startswith("opr_il_")}
    orr = {int(n.split("_")[-1]): from_npz(z, n, sym) for n in names if n.startswith("opr_ir_")}
    return z, m, psi, hl, hr, ol, orr


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_oracle_heff_matches_reference(path):
    z, m, psi, hl, hr, ol, orr = _load_heff_case(path)
    out = heff_apply(psi, hl, hr, ol, orr, m["hmap"], m["coup"], m["il"], m["ir"], m["ns"])
    ref = from_npz(z, "hpsi", m["sym"])
    assert set(out.blocks) == set(ref.blocks)
    scale = np.abs(ref.flat()).max()
    for k in ref.blocks:
        np.testing.assert_allclose(out.blocks[k], ref.blocks[k], rtol=0, atol=1e-13 * scale)


def test_cg_known_values():
    # <1/2 1/2; 1/2 -1/2 | 0 0> = 1/sqrt(2), <1/2 1/2; 1/2 1/2 | 1 1> = 1
    assert abs(cgc.cg(1, 1, 1, -1, 0, 0) - 1 / np.sqrt(2)) < 1e-15
    assert abs(cgc.cg(1, 1, 1, 1, 2, 2) - 1.0) < 1e-15
    assert cgc.cg(1, 1, 1, 1, 0, 0) == 0.0
    # orthonormality of the CGC map (j1=1, j2=2)
    for j3 in (1, 3):
        c = cgc.make_cgc(1, 2, j3).reshape(-1, j3 + 1)
        np.testing.assert_allclose(c.T @ c, np.eye(j3 + 1), atol=1e-14)
