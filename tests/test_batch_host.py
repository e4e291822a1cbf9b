"""CPU: host-side logic of the batched API that needs no device: the halo
chunks of the pipelined stage."""
import numpy as np

from galaxyfinder_b200 import batch, synth


def test_chunk_cuts_cover_the_batch_in_balanced_contiguous_chunks():
    hb = synth.catalogue(seed=synth.SEED_BASE + 5, nhalo=300, nmin=100, nmax=20000)
    for nchunk in (1, 3, 8, 16):
        cuts = batch.chunk_cuts(hb.pstart, nchunk)
        assert cuts[0] == 0 and cuts[-1] == hb.nhalo
        assert all(a < b for a, b in zip(cuts, cuts[1:]))
        sizes = np.diff(np.asarray(hb.pstart)[cuts])
        assert len(sizes) <= nchunk and sizes.sum() == hb.n
        # each chunk ends at the first halo boundary past its share, so it
        # exceeds n/nchunk by less than one halo
        biggest_halo = np.diff(hb.pstart).max()
        assert sizes.max() <= hb.n / nchunk + biggest_halo


def test_chunk_cuts_keep_a_dominant_halo_whole():
    ps = np.array([0, 10, 1_000_000, 1_000_010])  # one halo holds almost everything
    cuts = batch.chunk_cuts(ps, 8)
    assert cuts[0] == 0 and cuts[-1] == 3
    assert 1 in cuts or 2 in cuts
    np.testing.assert_array_equal(np.diff(ps[cuts]).sum(), ps[-1])
