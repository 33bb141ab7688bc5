"""The serving loop on the GPU: every request's energy is the same served
alone (one slot) and in the mix (three slots, overlapping on the device), and
equal to a direct solve; in the 3xTF32 form it matches FP64 to 1e-8 (four
sweeps at krylovdim 3 are not converged, so the two forms' truncations may
differ slightly)."""
import pytest

from sparsebackends_b200 import serving

pytestmark = pytest.mark.gpu


def test_alone_and_in_the_mix():
    reqs = serving.random_requests(6, seed=11, n_range=(8, 14), chi_range=(8, 24))
    stream = serving.poisson_arrivals(reqs, rate=40.0, seed=4)
    alone = serving.Server(slots=1).run(stream)
    mixed = serving.Server(slots=3).run(stream)
    assert [r.energy for r in alone] == [r.energy for r in mixed]
    assert max(r.slot for r in mixed) >= 1  # more than one slot was used
    srv = serving.Server(slots=1)
    for r, res in zip(reqs, alone):
        assert srv.solve(r, 0) == res.energy
    tc = serving.Server(slots=3, precision="tf32x3").run(stream)
    for a, b in zip(alone, tc):
        assert abs(a.energy - b.energy) <= 1e-8 * abs(a.energy), (a, b)

