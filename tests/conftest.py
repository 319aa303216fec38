"""pytest configuration: the `gpu` marker and shared fixture helpers."""
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "symmetry-adapted-dmrg-library_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def centre_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "centre_*.npz")))


def sweep_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "sweeps_*.npz")))


def fixture_tensor(z, prefix):
    """BlockTensorData (binding type) for tensor `prefix` of a golden npz."""
    import sadmrg
    nmom = [int(x) for x in z[prefix + "__nmom"]]
    q = [int(x) for x in z[prefix + "__q"]]
    d = [int(x) for x in z[prefix + "__d"]]
    qs, ds, o = [], [], 0
    for n in nmom:
        qs.append(q[o:o + n]); ds.append(d[o:o + n]); o += n
    return sadmrg.BlockTensorData([int(x) for x in z[prefix + "__dirs"]], qs, ds, int(z[prefix + "__locspin"]),
                                  np.array(z[prefix + "__blocks"], np.int64), np.array(z[prefix + "__data"]))


def tensor_names(z):
    return [k[:-6] for k in z.files if k.endswith("__dirs")]
