"""sgfd_energy_noalloc, the energy audit for callers that cannot let the
library allocate device memory while they run (their device memory belongs
to another allocator, or their footprint was fixed at start-up): its partial
sums live in a fixed array inside libsgfd.so instead of a cudaMalloc'd
buffer.  Checked through the C ABI against sgfd_energy, on two calls in a
row with steps between them, for its size limit, and on a fresh handle that
it makes no device allocation of its own.  Collected last, so a run that
stops at the first failure has run every other test first."""
import numpy as np
import pytest

from helpers import make_solver
import sgfd
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu

RTOL = 1e-10   # the tolerance of the energy audit tests


@pytest.mark.parametrize("region", [sgfd.REGION_COMPUTED, sgfd.REGION_INTERIOR, sgfd.REGION_PML],
                         ids=["computed", "interior", "pml"])
def test_noalloc_energy_matches_energy_on_two_calls(region):
    w = wl.small_random_case(nx=47, ny=41, nz=39, pml=6, nt=60)
    with make_solver(w) as s:
        for stop in (30, 60):                 # two calls in a row, the field changing between them
            s.run(stop - 30, 30)
            got = s.energy_noalloc(region)
            want = s.energy(region)
            assert want[0] > 0 and want[1] > 0
            np.testing.assert_allclose(got, want, rtol=RTOL)
        # another partial-sum block count within the limit sums in another order
        np.testing.assert_allclose(s.energy_noalloc(region, nblocks=97), want, rtol=RTOL)


def test_noalloc_energy_rejects_more_blocks_than_the_static_scratch_holds():
    w = wl.small_random_case(nt=10)
    with make_solver(w) as s:
        s.run(0, 10)
        np.testing.assert_allclose(s.energy_noalloc(0, nblocks=2047), s.energy(0), rtol=RTOL)
        with pytest.raises(sgfd.SgfdError) as e:
            s.energy_noalloc(0, nblocks=2048)
        assert e.value.code == sgfd.ERR_INVALID and "static scratch" in str(e.value)
        with pytest.raises(sgfd.SgfdError):
            s.energy_noalloc(5)


def test_noalloc_energy_makes_no_device_allocation_on_a_fresh_handle():
    """On a handle that never ran sgfd_energy (whose first call allocates the
    partial sums), sgfd_energy_noalloc leaves the handle's allocation count
    where it was, across two calls; sgfd_energy afterwards does allocate,
    which shows that the count sees such an allocation."""
    w = wl.small_random_case(nx=40, ny=36, nz=34, pml=5, nt=40)
    with make_solver(w) as s:
        s.run(0, 20)
        s.synchronize()
        before = s.device_allocations()
        first = s.energy_noalloc(sgfd.REGION_COMPUTED)
        s.run(20, 20)
        second = s.energy_noalloc(sgfd.REGION_COMPUTED)
        assert s.device_allocations() == before
        assert first[0] > 0 and second[0] > 0 and first != second
        want = s.energy(sgfd.REGION_COMPUTED)
        assert s.device_allocations() == before + 1
        np.testing.assert_allclose(second, want, rtol=RTOL)
