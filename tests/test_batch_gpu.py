"""GPU checks of the batch runner: maps lit side by side by several workers
give the same LIGHTING lumps, lightofs and ray counts as the single-map
calls, byte for byte, whatever the worker count and the tuned launch shape;
a map that fails leaves the others' lumps intact and the batch usable."""
import dataclasses

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import batch as B, lighting as L, roomgrid as rg

pytestmark = pytest.mark.gpu


def _worlds():
    small = [rg.config_batch(i, seed=5) for i in range(64)]
    picks = [c for c in small if c.side <= 3][:3]
    assert len(picks) == 3
    return [rg.generate(c) for c in picks] + [rg.generate(rg.config_3x3(seed=2))]


@pytest.fixture(scope="module")
def maps_and_singles():
    worlds = _worlds()
    maps = [B.map_inputs(worlds[0]), B.map_inputs(worlds[1], bounce=False),
            B.map_inputs(worlds[2], extra_passes=0), B.map_inputs(worlds[3], threshold=0.1)]
    singles = []
    for w, m in zip(worlds, maps):
        st = L.LightingStage(w, m.inputs)
        if m.extra_passes >= 0:
            st.set_extra_passes(m.extra_passes)
        if m.bounced:
            st.upload_bounce(m.reflectivity, m.pvs_offsets, m.pvs_clusters, bounces=m.bounces,
                             threshold=m.threshold)
        lump, ofs, ps = st.light_pass()
        bs = st.bounce_stats() if m.bounced else None
        singles.append((lump.copy(), ofs.copy(), ps.visibility_rays + ps.sky_rays,
                        (bs.transfer_rays, bs.transfers, bs.bounces) if bs else None))
        st.close()
    return maps, singles


def _same(results, singles):
    for k, (r, (lump, ofs, rays, bounce)) in enumerate(zip(results, singles)):
        assert r.status == 0, (k, r.error)
        assert np.array_equal(r.lighting, lump), k
        assert np.array_equal(r.lightofs, ofs), k
        assert r.pass_stats.visibility_rays + r.pass_stats.sky_rays == rays, k
        if bounce is not None:
            b = r.bounce_stats
            assert (b.transfer_rays, b.transfers, b.bounces) == bounce, k


def test_batch_lumps_equal_single_map_lumps(maps_and_singles):
    maps, singles = maps_and_singles
    with B.LightingBatch(workers=3) as batch:
        results, st = batch.run(maps)
        _same(results, singles)
        assert st.maps == 4 and st.failed == 0 and st.workers == 3
        assert st.lighting_bytes == sum(len(s[0]) for s in singles)
        assert len({r.worker for r in results}) >= 2           # the queue was shared
        # Again on the same contexts (re-uploads over the previous maps'
        # tables), and with one worker: the same bytes.
        _same(batch.run(maps)[0], singles)
        _same(batch.run(maps, workers=1)[0], singles)


def test_autotune_keeps_the_bytes(maps_and_singles):
    maps, singles = maps_and_singles
    with B.LightingBatch(workers=2) as batch:
        w, block, secs = batch.autotune(maps)
        assert w in (1, 2) and block in (32, 64, 128)
        assert set(secs) == {1, 2} and all(s > 0 for s in secs.values())
        results, st = batch.run(maps)
        assert st.workers == w and st.block == block
        _same(results, singles)


def test_a_failing_map_leaves_the_others(maps_and_singles):
    maps, singles = maps_and_singles
    bad_inputs = dataclasses.replace(maps[0].inputs, faces=maps[0].inputs.faces.copy())
    bad_inputs.faces["flags"][0] |= 0x0800            # a bump-mapped face: unsupported by the bounce
    bad = dataclasses.replace(maps[0], inputs=bad_inputs)
    with B.LightingBatch(workers=2) as batch:
        results, st = batch.run([maps[1], bad, maps[2]], raise_on_error=False)
        assert st.failed == 1 and results[1].status == -6 and "bump" in results[1].error.lower()
        _same([results[0], results[2]], [singles[1], singles[2]])
        with pytest.raises(NotImplementedError):
            batch.run([bad])
        _same(batch.run(maps)[0], singles)
