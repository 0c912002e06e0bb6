"""GPU parity of the bounce against the oracle's restatement of the
reference's PatchLighting, VisMatrix, FormFactors, Radiosity and
FinalLightFace.BuildPatchRadial.

The bar is bit-exact: every transfer (source and weight bits), every
patch's direct and bounced light, the number of bounces the stop rule runs,
and the LIGHTING lump's bytes."""
import numpy as np
import pytest

import fixtures
from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg, tracer as T

pytestmark = pytest.mark.gpu


def _stage(cfg, threshold=1.0, bounces=100):
    w = rg.generate(cfg)
    inp = L.prepare(w)
    st = L.LightingStage(w, inp)
    off, lst = L.pvs_lists(w)
    st.upload_bounce(L.face_reflectivity(w), off, lst, bounces=bounces, threshold=threshold)
    return w, inp, st


def _oracle(O, w, inp, threshold=1.0, bounces=100):
    tree = O.kd_build(w.tri_verts, w.tri_ids)
    off, lst = L.pvs_lists(w)
    return O.Bounce(tree, inp.faces, inp.verts, inp.samples, inp.face_first, L.face_reflectivity(w), off, lst,
                    bounces=bounces, threshold=threshold)


def _sample_light(st):
    s, _ = st.direct()
    return np.concatenate([s["lighting"], s["direct_sun_amount"][:, None]], 1)


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_detmath_asin_and_pow_match_goldens():
    import ctypes
    tr = T.CudaRayTracer(T.make_triangles(np.zeros((1, 9), np.float32), np.zeros(1, np.int32)))
    lib = T.load_library()
    lib.vrad_detmath.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    for fn, name in ((0, "Asin"), (1, "Pow")):
        a, b, e = fixtures.detmath(name)
        out = np.zeros(len(a), np.float32)
        open_ = ctypes.c_int64()
        rc = lib.vrad_detmath(tr._ctx, fn, a.ctypes.data, b.ctypes.data, out.ctypes.data, len(a), ctypes.byref(open_))
        assert rc == 0
        got = out.view(np.uint32)
        bad = np.flatnonzero(got != e)
        assert len(bad) == 0, (name, [(hex(a[i]), hex(b[i]), hex(got[i]), hex(e[i])) for i in bad[:6]])
    tr.close()


@pytest.mark.parametrize("threshold", [1.0, 0.1], ids=["stock-1.0", "config-0.1"])
def test_3x3_bounce_bit_exact(oracle_mod, threshold):
    w, inp, st = _stage(rg.config_3x3(seed=2), threshold=threshold)
    with st:
        lump, lightofs, _ = st.light_pass()
        bs = st.bounce_stats()
        total, direct = st.patch_light()
        off, tr = st.transfers()
        last = st.last_total()
        light = _sample_light(st)
    ob = _oracle(oracle_mod, w, inp, threshold=threshold)
    o_off, o_src, o_w, rays = ob.transfers()
    assert bs.transfer_rays == rays
    assert np.array_equal(off, o_off)
    assert np.array_equal(tr["patch"], o_src)
    assert np.array_equal(_bits(tr["weight"]), _bits(o_w))
    o_total, o_direct, o_bounces, o_added = ob.run(light)
    assert np.array_equal(_bits(direct), _bits(o_direct))
    assert bs.bounces == o_bounces and bs.bounces > 1
    assert np.array_equal(_bits(last), _bits(o_added))
    assert np.array_equal(_bits(total), _bits(o_total))
    want, want_ofs = ob.final(light)
    assert np.array_equal(lightofs, want_ofs)
    bad = np.flatnonzero(lump.view(np.uint32) != want.view(np.uint32))
    assert len(bad) == 0, f"{len(bad)} of {len(lump) // 4} RGBE words differ"
    # The bounce adds light.
    assert (total > 0).any() and bs.transfers == len(tr) > 0


def test_8x8_transfers_sampled_and_bounce_bit_exact(oracle_mod):
    w, inp, st = _stage(rg.config_8x8(seed=1))
    with st:
        lump, lightofs, _ = st.light_pass()
        bs = st.bounce_stats()
        total, direct = st.patch_light()
        off, tr = st.transfers()
        last = st.last_total()
        light = _sample_light(st)
    ob = _oracle(oracle_mod, w, inp)
    patches, _ = ob.patches()
    leaves = np.flatnonzero(patches["child1"] == -1)
    rng = np.random.default_rng(7)
    sub = np.sort(rng.choice(leaves, 400, replace=False))
    o_off, o_src, o_w, _ = ob.transfers(sub)
    for p in sub:
        a, b = off[p], off[p + 1]
        c, d = o_off[p], o_off[p + 1]
        assert np.array_equal(tr["patch"][a:b], o_src[c:d]), p
        assert np.array_equal(_bits(tr["weight"][a:b]), _bits(o_w[c:d])), p
    # The bounce itself over the device's transfers.
    ob.set_transfers(off, tr["patch"], tr["weight"])
    o_total, o_direct, o_bounces, o_added = ob.run(light)
    assert np.array_equal(_bits(direct), _bits(o_direct))
    assert bs.bounces == o_bounces
    assert np.array_equal(_bits(total), _bits(o_total))
    # CollectLight's sequential float total over the million leaves, as the
    # device's exact-sum kernel computes it when the fp64 bound is unsure.
    assert np.array_equal(_bits(last), _bits(o_added))
    want, want_ofs = ob.final(light)
    bad = np.flatnonzero(lump.view(np.uint32) != want.view(np.uint32))
    assert len(bad) == 0, f"{len(bad)} of {len(lump) // 4} RGBE words differ"


def test_bounce_pass_is_repeatable_and_device_entry_matches():
    import torch
    w, inp, st = _stage(rg.config_3x3(seed=2))
    with st:
        a, _, _ = st.light_pass()
        b, _, _ = st.light_pass()
        d = torch.zeros(len(a), dtype=torch.uint8, device="cuda")
        st.light_pass_device(d)
        torch.cuda.synchronize()
    assert np.array_equal(a, b)
    assert np.array_equal(d.cpu().numpy(), a)


def test_sample_runs_in_any_face_order_light_the_same_lump():
    """The world upload takes each face's samples as one contiguous run, the
    runs in any order of faces: an upload with the runs permuted lights the
    same lump, bounce included (supersampling off in both, since it needs
    the sample builder's own order)."""
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    off, lst = L.pvs_lists(w)
    refl = L.face_reflectivity(w)
    ff = inp.face_first
    order = np.random.default_rng(5).permutation(len(inp.faces))
    idx = np.concatenate([np.arange(ff[f], ff[f + 1]) for f in order])
    perm = L.LightingInputs(**{**inp.__dict__, "samples": inp.samples[idx].copy()})
    lumps, stats = [], []
    for i in (inp, perm):
        with L.LightingStage(w, i) as st:
            st.set_extra_passes(0)
            st.upload_bounce(refl, off, lst, threshold=1.0)
            lump, _, _ = st.light_pass()
            lumps.append(lump)
            stats.append(st.bounce_stats().bounces)
    assert stats[0] == stats[1] and stats[0] > 1
    assert np.array_equal(lumps[0], lumps[1])


def test_reupload_grows_the_patch_forest_ahead_and_keeps_the_lump():
    """A context that has bounced grows the next world's patch forest while
    the world uploads, with its last chop sizes; the bounce upload takes it
    when the sizes match and grows its own when they do not.  Either way the
    lump is a fresh context's, and a new reflectivity still applies."""
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    off, lst = L.pvs_lists(w)
    refl = L.face_reflectivity(w)
    dim = (refl * np.float32(0.5)).astype(np.float32)

    def fresh(r, max_chop):
        st = L.LightingStage(w, inp)
        st.upload_bounce(r, off, lst, max_chop=max_chop)
        lump = st.light_pass()[0].copy()
        st.close()
        return lump

    want = {(0, 4.0): fresh(refl, 4.0), (0, 8.0): fresh(refl, 8.0), (1, 4.0): fresh(dim, 4.0)}
    assert not np.array_equal(want[(0, 4.0)], want[(0, 8.0)])
    st = L.LightingStage(w, inp)
    st.upload_bounce(refl, off, lst)
    for which, chop in ((0, 4.0), (0, 8.0), (0, 8.0), (1, 4.0), (0, 4.0)):
        st.upload_world(inp)
        st.upload_bounce(dim if which else refl, off, lst, max_chop=chop)
        assert np.array_equal(st.light_pass()[0], want[(which, chop)]), (which, chop)
    st.close()


def test_direct_gather_queued_at_the_world_upload_lights_the_same_lump():
    """The world upload queues the direct gather ahead (it overlaps the
    bounce upload); the next host-buffer light pass takes it.  The lump is
    the one a pass that gathers itself writes, and a setting changed after
    the upload (the supersampling passes) drops the queued gather."""
    import torch
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    off, lst = L.pvs_lists(w)
    refl = L.face_reflectivity(w)
    st = L.LightingStage(w, inp)
    st.upload_bounce(refl, off, lst)
    ahead, _, ps = st.light_pass()                   # takes the gather queued by the world upload
    ahead = ahead.copy()
    d = torch.empty(len(ahead), dtype=torch.uint8, device="cuda")
    st.light_pass_device(d)                          # gathers itself
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), ahead)
    st.upload_world(inp)
    st.set_extra_passes(0)                           # after the upload: the queued gather is dropped
    st.upload_bounce(refl, off, lst)
    noextra, _, ps0 = st.light_pass()
    assert ps0.extra_passes_run == 0 and ps.extra_passes_run > 0
    st.close()
    st = L.LightingStage(w, inp)
    st.set_extra_passes(0)
    st.upload_world(inp)                             # queued with no extra passes
    st.upload_bounce(refl, off, lst)
    assert np.array_equal(st.light_pass()[0], noextra)
    st.close()
