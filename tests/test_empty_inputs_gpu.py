"""Zero-length batches on every path, as the reference's allocating wrappers allow
them (an empty batch gives an empty output and zero parameter gradients)."""
import numpy as np
import pytest
import torch

import aok_b200 as aok
from helpers import to_np

W = aok.workloads
pytestmark = pytest.mark.gpu


def test_empty_inputs_every_path():
    none = np.zeros((3, 0))
    # GaussianBasis path: 2C and 3C
    bc = aok.compile_basis([aok.CartesianShell(0, np.array([1.0]), np.array([1.0])),
                            aok.CartesianShell(1, np.array([0.6, 0.4]), np.array([0.9, 0.3]))])
    L0 = aok.Length(none, "bohr")
    assert tuple(aok.batch_overlap(bc, L0, L0).shape) == (4, 4, 0)
    assert tuple(aok.batch_overlap_3c(bc, L0, L0, L0).shape) == (4, 4, 4, 0)
    assert tuple(aok.batch_overlap_3c(bc, L0, L0, L0, FT=torch.float32).shape) == (4, 4, 4, 0)

    # species-aware 2C pullback: no pairs, zero (zeta, D) gradients
    b = W.config2_basis()
    orb = aok.orbitals_from_species_basis(b)
    ps, st = aok.initialparameters(orb), aok.initialstates(orb)
    X0 = aok.PStates(none, [])
    N = b.nbf_total
    g = aok.overlap_pullback_ps(np.zeros((N, N, 0)), orb, X0, X0, ps, st)
    assert np.all(to_np(g["Rnl"]["zeta"]) == 0) and np.all(to_np(g["Rnl"]["D"]) == 0)
    assert to_np(g["Rnl"]["zeta"]).shape == b.zeta.shape

    # orbital evaluation and its pullback
    b1 = W.config1_basis()
    orb1 = aok.orbitals_from_species_basis(b1)
    nOrb = len(orb1)
    assert tuple(aok.evaluate(orb1, none).shape) == (0, nOrb)
    P, dP = aok.evaluate_ed(orb1, none)
    assert tuple(P.shape) == (0, nOrb) and tuple(dP.shape) == (0, nOrb, 3)
    ps1, st1 = aok.initialparameters(orb1), aok.initialstates(orb1)
    g1 = aok.evaluate_pullback_ps(np.zeros((0, nOrb)), orb1, X0, ps1, st1)
    assert np.all(to_np(g1["Rnl"]["zeta"]) == 0) and np.all(to_np(g1["Rnl"]["D"]) == 0)
