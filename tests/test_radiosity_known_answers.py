"""The bounce against the reference's own radiosity tests
(src/SourceSharp.Tests/MapTools/Rad/Bounce/RadiosityTests.cs) on the same
scene: the BounceBox (Bounce/BounceBox.cs over Light/DirectLightTests.cs's
LightBox and Light/LightTestMap.cs), a closed 256-unit box of six faces
(floor, ceiling, four walls) in one cluster that sees itself, lightmap scale
16, texture axes and reflectivity 0.5 as LightTestMap gives them, each face
a shadow caster of two triangles, and one "light" at (128 128 128) with
"_light" "255 255 255 200".

Each property the reference asserts is checked on the oracle (CPU) and on
the device through the C ABI (vrad_bounce_upload, vrad_light_pass,
vrad_bounce_patch_light, vrad_bounce_transfers, vrad_bounce_last_total),
and the device's patch light and bounce count against the oracle's bits.
The reference's UnevenChildren and bump-mapped variants change patch
fields in memory, which this ABI does not expose; those cases are not
restated.
"""
import types

import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, lights as LT, workload as wl

S = 256.0
TRACE_ID_SKY = 0x01000000


def _box(ceiling_sky=False, occluder=False):
    # LightBox.Map: (texinfo s axis, t axis, normal, corners) per face.
    floor_st = ((1, 0, 0), (0, -1, 0))
    wall_st = ((0, 1, 0), (0, 0, -1))
    wallx_st = ((1, 0, 0), (0, 0, -1))
    faces_def = [
        (floor_st, (0, 0, 1), [(0, S, 0), (S, S, 0), (S, 0, 0), (0, 0, 0)]),          # AddFloor up
        (floor_st, (0, 0, -1), [(0, 0, S), (S, 0, S), (S, S, S), (0, S, S)]),         # AddFloor down
        (wall_st, (1, 0, 0), [(0, 0, S), (0, S, S), (0, S, 0), (0, 0, 0)]),
        (wall_st, (-1, 0, 0), [(S, S, S), (S, 0, S), (S, 0, 0), (S, S, 0)]),
        (wallx_st, (0, 1, 0), [(S, 0, S), (0, 0, S), (0, 0, 0), (S, 0, 0)]),
        (wallx_st, (0, -1, 0), [(0, S, S), (S, S, S), (S, S, 0), (0, S, 0)]),
    ]
    faces = np.zeros(len(faces_def), L.FACE_DTYPE)
    verts, tris, ids = [], [], []
    for i, ((sa, ta), n, corners) in enumerate(faces_def):
        c = np.array(corners, np.float32)
        s = np.array(list(np.float32(sa) * np.float32(1 / 16)) + [0], np.float32)
        t = np.array(list(np.float32(ta) * np.float32(1 / 16)) + [0], np.float32)
        sv = [np.float32(np.float32(np.float32(p[0] * s[0]) + np.float32(p[1] * s[1])) + np.float32(p[2] * s[2])) + s[3]
              for p in c]
        tv = [np.float32(np.float32(np.float32(p[0] * t[0]) + np.float32(p[1] * t[1])) + np.float32(p[2] * t[2])) + t[3]
              for p in c]
        mins = (int(np.floor(min(sv))), int(np.floor(min(tv))))
        faces[i]["normal"] = n
        faces[i]["dist"] = np.float32(np.dot(np.float32(n), c[0]))
        faces[i]["lightmap_vecs"][0] = s
        faces[i]["lightmap_vecs"][1] = t
        faces[i]["lightmap_mins"] = mins
        faces[i]["lightmap_size"] = (int(np.ceil(max(sv))) - mins[0], int(np.ceil(max(tv))) - mins[1])
        faces[i]["first_vertex"] = len(verts)
        faces[i]["num_vertices"] = 4
        sky = ceiling_sky and i == 1
        faces[i]["flags"] = 0x0004 if sky else 0
        verts.extend(corners)
        ident = TRACE_ID_SKY if sky else 0
        tris += [np.concatenate([c[0], c[1], c[2]]), np.concatenate([c[0], c[2], c[3]])]
        ids += [ident, ident]
    if occluder:
        # AnOccluderRemovesTransfers: map.AddOccluder((8 8 128) (248 8 128)
        # (248 248 128) (8 248 128)), a caster that is no face.
        c = np.array([(8, 8, 128), (248, 8, 128), (248, 248, 128), (8, 248, 128)], np.float32)
        tris += [np.concatenate([c[0], c[1], c[2]]), np.concatenate([c[0], c[2], c[3]])]
        ids += [0, 0]
    verts = np.array(verts, np.float32)
    samples, first = L.build_samples(faces, verts)
    ls = LT.build([LT.entity(("classname", "worldspawn")),
                   LT.entity(("classname", "light"), ("origin", "128 128 128"), ("_light", "255 255 255 200"))])
    lights = LT.to_records(ls.active, L.LIGHT_DTYPE)
    inp = L.LightingInputs(faces, verts, samples, first, lights, np.array([0, 1], np.int32), np.array([0], np.int32),
                           wl.ambient_directions().astype(np.float32), np.zeros((0, 3), np.float32))
    world = types.SimpleNamespace(tri_verts=np.stack(tris).astype(np.float32), tri_ids=np.array(ids, np.int32))
    refl = np.full((len(faces), 3), 0.5, np.float32)
    return world, inp, refl


PVS = (np.array([0, 1], np.int32), np.array([0], np.int32))
NO_SELF = (np.array([0, 0], np.int32), np.array([], np.int32))   # BounceBox.Map(seesItself: false)


def _oracle(O, world, inp, refl, bounces, threshold=1.0, pvs=PVS):
    tree = O.kd_build(world.tri_verts, world.tri_ids)
    light = O.direct(tree, inp.faces, inp.samples, inp.face_first, inp.lights, inp.cluster_offsets,
                     inp.cluster_lights, inp.sky_directions, verts=inp.verts)
    ob = O.Bounce(tree, inp.faces, inp.verts, inp.samples, inp.face_first, refl, *pvs, bounces=bounces,
                  threshold=threshold)
    patches, _ = ob.patches()
    off, src, w, rays = ob.transfers()
    total, direct, n, added = ob.run(light)
    return dict(patches=patches, off=off, src=src, w=w, total=total, direct=direct, bounces=n, last=added,
                rays=rays)


def _device(world, inp, refl, bounces, threshold=1.0, pvs=PVS):
    with L.LightingStage(world, inp) as st:
        st.upload_bounce(refl, *pvs, bounces=bounces, threshold=threshold)
        st.light_pass()
        total, direct = st.patch_light()
        off, tr = st.transfers()
        bs = st.bounce_stats()
        last = st.last_total() if bs.bounces > 0 else None
    patches, _ = L.build_patches(inp.faces, inp.verts, refl)
    return dict(patches=patches, off=off, src=tr["patch"], w=tr["weight"], total=total, direct=direct,
                bounces=bs.bounces, last=last, rays=bs.transfer_rays, blocked=getattr(bs, "blocked_rays", None))


def _leaves(r):
    p = r["patches"]
    return np.flatnonzero((p["child1"] == -1) & (p["sky"] == 0))


def _gathered(r, refl_of_patch, j):
    """GatherLight's sum for patch j: (emit * reflectivity) * weight over its
    list, in list order, emit being the direct light after
    MoveDirectLightToEmission."""
    acc = np.zeros(3, np.float32)
    for k in range(r["off"][j], r["off"][j + 1]):
        s = r["src"][k]
        e = r["direct"][s] * refl_of_patch[s]
        acc = (acc + (e * r["w"][k]).astype(np.float32)).astype(np.float32)
    return acc


def _check_one_bounce(r):
    refl_of_patch = r["patches"]["reflectivity"].astype(np.float32)
    leaves = _leaves(r)
    assert (r["direct"][leaves] > 0).any()
    # A flat patch sums emit x reflectivity x transfer in list order, and
    # after one bounce its total is exactly that (bounced light only: the
    # direct light was moved out first).
    for j in leaves:
        assert np.array_equal(r["total"][j].view(np.uint32), _gathered(r, refl_of_patch, j).view(np.uint32)), j
    # CollectLight's total is the leaves' new emission summed in reverse
    # patch order.
    acc = np.zeros(3, np.float32)
    for i in leaves[::-1]:
        acc = (acc + r["total"][i]).astype(np.float32)
    assert np.array_equal(np.asarray(r["last"], np.float32).view(np.uint32), acc.view(np.uint32))
    # A parent is its children, area weighted.
    p = r["patches"]
    for i in np.flatnonzero(p["child1"] != -1):
        c1, c2 = p["child1"][i], p["child2"][i]
        a1, a2 = p["area"][c1], p["area"][c2]
        s1 = np.float32(a1 / np.float32(a1 + a2))
        s2 = np.float32(a2 / np.float32(a1 + a2))
        want = (r["total"][c1] * s1).astype(np.float32) + (r["total"][c2] * s2).astype(np.float32)
        assert np.array_equal(r["total"][i].view(np.uint32), want.astype(np.float32).view(np.uint32)), i


def test_oracle_one_bounce_properties(oracle_mod):
    world, inp, refl = _box()
    r = _oracle(oracle_mod, world, inp, refl, bounces=1)
    assert r["bounces"] == 1
    _check_one_bounce(r)


def test_oracle_stop_rules(oracle_mod):
    world, inp, refl = _box()
    assert _oracle(oracle_mod, world, inp, refl, bounces=3)["bounces"] == 3
    r = _oracle(oracle_mod, world, inp, refl, bounces=100)
    assert 3 < r["bounces"] < 100 and (r["last"] < 1).all()
    r0 = _oracle(oracle_mod, world, inp, refl, bounces=0)
    assert r0["bounces"] == 0 and not r0["total"].any()


def test_oracle_sky_patch_emits_nothing(oracle_mod):
    world, inp, refl = _box(ceiling_sky=True)
    r = _oracle(oracle_mod, world, inp, refl, bounces=100)
    sky = np.flatnonzero(r["patches"]["sky"] != 0)
    assert len(sky) and not r["total"][sky].any()


@pytest.mark.gpu
def test_device_one_bounce_properties_and_oracle_bits(oracle_mod):
    world, inp, refl = _box()
    r = _device(world, inp, refl, bounces=1)
    assert r["bounces"] == 1
    _check_one_bounce(r)
    o = _oracle(oracle_mod, world, inp, refl, bounces=1)
    for k in ("total", "direct"):
        assert np.array_equal(r[k].view(np.uint32), o[k].view(np.uint32)), k


@pytest.mark.gpu
def test_device_stop_rules(oracle_mod):
    world, inp, refl = _box()
    assert _device(world, inp, refl, bounces=3)["bounces"] == 3
    r = _device(world, inp, refl, bounces=100)
    o = _oracle(oracle_mod, world, inp, refl, bounces=100)
    assert r["bounces"] == o["bounces"] and (r["last"] < 1).all()
    assert np.array_equal(np.asarray(r["last"], np.float32).view(np.uint32), o["last"].view(np.uint32))
    r0 = _device(world, inp, refl, bounces=0)
    assert r0["bounces"] == 0 and not r0["total"].any()


@pytest.mark.gpu
def test_device_sky_patch_emits_nothing():
    world, inp, refl = _box(ceiling_sky=True)
    r = _device(world, inp, refl, bounces=100)
    sky = np.flatnonzero(r["patches"]["sky"] != 0)
    assert len(sky) and not r["total"][sky].any()


# ---- VisMatrixTests (Tests/MapTools/Rad/Bounce/VisMatrixTests.cs) on the box

def _check_transfer_lists(r):
    p = r["patches"]
    counts = np.diff(r["off"])
    leaves = set(_leaves(r).tolist())
    assert counts.sum() > 0
    for j in range(len(p)):
        if j not in leaves:
            assert counts[j] == 0, j                 # OnlyClusterChildrenHaveTransfers
            continue
        src = r["src"][r["off"][j]:r["off"][j + 1]]
        assert not (p["face"][src] == p["face"][j]).any(), j   # NoPatchTakesLightFromItsOwnFace
        acc = np.float32(0)
        for x in r["w"][r["off"][j]:r["off"][j + 1]]:
            acc = np.float32(acc + x)
        assert acc <= np.float32(1.0001), (j, acc)    # EveryListSumsToAtMostOne
    floor = [j for j in leaves if p["face"][j] == 0]
    assert all((p["face"][r["src"][r["off"][j]:r["off"][j + 1]]] == 1).any() for j in floor)  # floor sees ceiling


def _visibility_cases(run):
    world, inp, refl = _box()
    open_ = run(world, inp, refl)
    _check_transfer_lists(open_)
    world, inp, refl = _box(occluder=True)
    shut = run(world, inp, refl)
    assert len(shut["src"]) < len(open_["src"])       # AnOccluderRemovesTransfers
    world, inp, refl = _box()
    none = run(world, inp, refl, pvs=NO_SELF)
    assert len(none["src"]) == 0 and none["rays"] == 0  # APvsThatExcludesTheClusterMakesNoTransfers
    return open_


def test_oracle_transfer_lists(oracle_mod):
    _visibility_cases(lambda w, i, r, pvs=PVS: _oracle(oracle_mod, w, i, r, bounces=1, pvs=pvs))


@pytest.mark.gpu
def test_device_transfer_lists(oracle_mod):
    d = _visibility_cases(lambda w, i, r, pvs=PVS: _device(w, i, r, bounces=1, pvs=pvs))
    world, inp, refl = _box()
    o = _oracle(oracle_mod, world, inp, refl, bounces=1)
    assert np.array_equal(d["off"], o["off"]) and np.array_equal(d["src"], o["src"])
    assert np.array_equal(d["w"].view(np.uint32), o["w"].view(np.uint32))
