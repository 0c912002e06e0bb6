"""GPU parity of the full light pass with -bounce 0 (vrad_light_pass): the
LIGHTING lump's bytes against the oracle's restatement of FinalLightFace
over the oracle's own direct gather.  The bar is byte-identical: every
RGBE word of every luxel and every per-face median."""
import numpy as np
import pytest

from hl2sdk_tools_sharp_b200 import lighting as L, roomgrid as rg

pytestmark = pytest.mark.gpu


def test_3x3_lighting_lump_byte_identical(oracle_mod):
    w = rg.generate(rg.config_3x3(seed=2))
    inp = L.prepare(w)
    with L.LightingStage(w, inp) as st:
        lump, lightofs, stats = st.light_pass()
    tree = oracle_mod.kd_build(w.tri_verts, w.tri_ids)
    light = oracle_mod.direct(tree, inp.faces, inp.samples, inp.face_first, inp.lights, inp.cluster_offsets,
                              inp.cluster_lights, inp.sky_directions, verts=inp.verts)
    want, want_ofs = oracle_mod.final(inp.faces, inp.verts, inp.samples, inp.face_first, light)
    assert np.array_equal(lightofs, want_ofs)
    assert len(lump) == len(want) == stats.lighting_bytes
    bad = np.flatnonzero(lump.view(np.uint32) != want.view(np.uint32))
    assert len(bad) == 0, f"{len(bad)} of {len(lump) // 4} RGBE words differ"
    # Sanity: most luxels are lit, exponents are in range.
    assert (lump.view(np.uint32) != 0).mean() > 0.5
    assert stats.luxels == sum((f[0] + 1) * (f[1] + 1) for f in inp.faces["lightmap_size"])


def test_8x8_final_pass_byte_identical_on_gpu_samples(oracle_mod):
    # The whole 8x8 map: the oracle's final pass fed the GPU's sample light
    # (itself checked bit for bit by test_direct_gpu), against the GPU's lump.
    w = rg.generate(rg.config_8x8(seed=1))
    inp = L.prepare(w)
    with L.LightingStage(w, inp) as st:
        lump, lightofs, stats = st.light_pass()
        samples, _ = st.direct()
    light = np.concatenate([samples["lighting"], samples["direct_sun_amount"][:, None]], 1)
    want, want_ofs = oracle_mod.final(inp.faces, inp.verts, inp.samples, inp.face_first, light)
    assert np.array_equal(lightofs, want_ofs)
    bad = np.flatnonzero(lump.view(np.uint32) != want.view(np.uint32))
    assert len(bad) == 0, f"{len(bad)} of {len(lump) // 4} RGBE words differ"
    assert stats.final_ms > 0 and stats.direct_ms > stats.final_ms


def test_light_pass_device_matches_host():
    import torch
    w = rg.generate(rg.config_3x3(seed=2))
    with L.LightingStage(w) as st:
        lump, _, _ = st.light_pass()
        d = torch.zeros(len(lump), dtype=torch.uint8, device="cuda")
        st.light_pass_device(d)
        torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), lump)
