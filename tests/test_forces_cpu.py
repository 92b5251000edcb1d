"""Band-energy gradient references on the CPU: the Hellmann-Feynman sum over
the oracle's dH/dPOS, dS/dPOS agrees with central differences of E.  This
pins the packed-state conventions the GPU adjoint (lapw1gpu_forces) relies
on, with no GPU."""
import numpy as np
import pytest

from hack_wein2k_b200 import synth
from tests import force_ref as FR


@pytest.mark.parametrize("kind", ["lo", "ins"])
def test_hellmann_feynman_matches_band_energy_fd(kind):
    p = synth.small_case(kind)
    w, _ = FR.eigh(p)
    nb, gap = FR.gapped_nb(w)
    assert gap > 1e-3
    g = FR.hf_gradient(p, nb)
    scale = np.abs(g).max()
    assert scale > 1e-3
    for a, c in [(0, 0), (1, 2), (2, 1)]:
        fd = FR.fd_band_energy(p, nb, a, c)
        assert abs(fd - g[a, c]) <= 2e-6 * scale, (a, c, fd, g[a, c])


def test_gradient_is_translation_invariant():
    """A common shift t of all atoms multiplies every element (J, I) of H
    and S by exp(2 pi i (KZZ_J - KZZ_I) . t): the same unitary diagonal
    similarity on both, which leaves the eigenvalues unchanged, so the
    gradients of all atoms sum to zero.  The "ins" case has no warped
    interstitial potential, the one input that does not move with the atoms."""
    p = synth.small_case("ins")
    w, _ = FR.eigh(p)
    nb, _ = FR.gapped_nb(w)
    g = FR.hf_gradient(p, nb)
    assert np.abs(g.sum(axis=0)).max() <= 1e-6 * np.abs(g).max()
