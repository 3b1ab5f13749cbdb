"""ymrt_b200 against the reference's own CUDA kernels, rebuilt for sm_100a.

The reference's stage kernels (src/Shading.cu Ray_generation_path_tracing,
Ray_trace_path_tracing, Ray_shading_path_tracing) run on the same device,
driven by the reference's wave loop (oracle/ref_gpu_harness.cu), on the same
scene files and Halton tables.

* "exact" build (no FMA contraction, IEEE division and square root -- the
  flags ymrt_b200 is built with): per-sample radiance must agree within 1e-5
  relative on every pixel (both sides use CUDA's own math library); a pixel
  that differed would be replayed and classified in the failure message.
* the reference's default build (nvcc defaults, as its CMake build uses):
  FMA contraction changes last bits and so some sampled directions, so only
  the converged image is compared (RMSE at 16 spp).

The reference's kernels run only on scenes whose BVHs fit their 32-entry
traversal stacks (checked on the CPU by test_scene_host.py).
"""
import numpy as np
import pytest

import divergence as D
import ymrt_b200 as Y

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refgpu(oracle):
    if not oracle.gpu_available(exact=True) or not oracle.gpu_available(exact=False):
        try:
            from oracle import build_ref
            build_ref.build_gpu(exact=True)
            build_ref.build_gpu(exact=False)
        except Exception as e:
            pytest.skip(f"device build of the reference unavailable: {e}")
    return oracle


def _pair(ctx, refgpu, path, perm, w, h, exact):
    ours = Y.Scene(ctx, Y.HostScene(path, w, h), perm)
    ref = refgpu.RefGpuScene(path, perm, w, h, exact=exact)
    return ours, ref


@pytest.mark.parametrize("frame", [1, 2])
def test_per_sample_cornell_vs_reference_cuda(ctx, refgpu, cornell_path, halton_perm, frame):
    ours, ref = _pair(ctx, refgpu, cornell_path, halton_perm, 256, 256, exact=True)
    ref.set_settings(spp=1, ray_depth=8)
    s = Y.default_setting(spp=1, ray_depth=8)
    a, _ = ours.render(s, frame)
    b = ref.render_frame(frame)
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_device_build(f"refcuda_cornell_f{frame}", ours, ref, s, frame, a, b)
    ours.close()
    ref.close()


def test_per_sample_instanced_tiles_vs_reference_cuda(ctx, refgpu, instanced_path, halton_perm):
    ours, ref = _pair(ctx, refgpu, instanced_path, halton_perm, 1920, 1080, exact=True)
    ref.set_settings(spp=1, ray_depth=12)
    tiles = (3600, 3760)
    s = Y.default_setting(spp=1, ray_depth=12)
    a, _ = ours.render(s, 1, tile_begin=tiles[0], tile_end=tiles[1])
    b = ref.render_frame(1, tile_begin=tiles[0], tile_end=tiles[1])
    covered = b[..., 3] > 0
    assert covered.sum() == (tiles[1] - tiles[0]) * 256
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_device_build("refcuda_instanced_tiles", ours, ref, s, 1, a, b, tiles[0], tiles[1], mask=covered)
    ours.close()
    ref.close()


@pytest.mark.parametrize("distant,volume", [(1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("frame", [1, 2])
def test_per_sample_volumetric_vs_reference_cuda(ctx, refgpu, volumetric_path, halton_perm, distant, volume, frame):
    ours, ref = _pair(ctx, refgpu, volumetric_path, halton_perm, 256, 256, exact=True)
    ref.set_settings(spp=1, ray_depth=8, distant_light=distant, volume=volume)
    s = Y.default_setting(spp=1, ray_depth=8, distant_light=bool(distant), volume=bool(volume))
    a, _ = ours.render(s, frame)
    b = ref.render_frame(frame)
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_device_build(f"refcuda_volumetric_d{distant}v{volume}_f{frame}", ours, ref, s, frame, a, b)
    ours.close()
    ref.close()


@pytest.mark.parametrize("volume", [0, 1])
def test_per_sample_spheres_vs_reference_cuda(ctx, refgpu, scene_dir, halton_perm, volume):
    """Sphere and Cube blocks: a glass and a metal sphere, a sphere light, a
    medium-filled boundary sphere around the camera and the built-in cube."""
    from ymrt_b200 import scenes
    path = scenes.scene_path("spheres", 0, scene_dir)
    ours, ref = _pair(ctx, refgpu, path, halton_perm, 256, 256, exact=True)
    ref.set_settings(spp=1, ray_depth=8, volume=volume)
    s = Y.default_setting(spp=1, ray_depth=8, volume=bool(volume))
    a, _ = ours.render(s, 2)
    b = ref.render_frame(2)
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_device_build(f"refcuda_spheres_v{volume}", ours, ref, s, 2, a, b)
    ours.close()
    ref.close()


@pytest.mark.parametrize("volume", [0, 1])
def test_per_sample_textured_vs_reference_cuda(ctx, refgpu, scene_dir, halton_perm, volume):
    """Procedural texture nodes on material parameters, as normal and bump
    maps and as media densities (the device harness uploads no image
    tiles, so image nodes are pinned against the host oracle only)."""
    from ymrt_b200 import scenes
    path = scenes.scene_path("textured", 0, scene_dir)
    ours, ref = _pair(ctx, refgpu, path, halton_perm, 256, 256, exact=True)
    ref.set_settings(spp=1, ray_depth=8, volume=volume)
    s = Y.default_setting(spp=1, ray_depth=8, volume=bool(volume))
    a, _ = ours.render(s, 1)
    b = ref.render_frame(1)
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_device_build(f"refcuda_textured_v{volume}", ours, ref, s, 1, a, b)
    ours.close()
    ref.close()


@pytest.mark.parametrize("scene,volume", [("cornell", 0), ("volumetric", 1), ("spheres", 1)])
def test_recorded_vertices_equal_the_reference_cuda(ctx, refgpu, scene_dir, halton_perm, scene, volume):
    """Every vertex that hits something, on 1 pixel in 61 of a 256x256
    frame: the ray, hit, throughput and received light that ymrt_b200's
    closest-hit stage leaves equal, bit for bit, what the reference's trace
    stage writes to its hit queue."""
    from ymrt_b200 import scenes
    path = scenes.scene_path(scene, 0, scene_dir)
    ours, ref = _pair(ctx, refgpu, path, halton_perm, 256, 256, exact=True)
    kw = dict(spp=1, ray_depth=8, distant_light=scene == "volumetric", volume=bool(volume))
    ref.set_settings(**{k: int(v) for k, v in kw.items()})
    s = Y.default_setting(**kw)
    pixels = np.arange(0, 256 * 256, 61)
    ra, _ = ours.record_paths(s, pixels, 3)
    rb, _ = ref.record_paths(pixels, 3)
    ra = ra[(ra["flags"] & 1) == 1]
    key_a = np.lexsort((ra["depth"], ra["pixel"]))
    key_b = np.lexsort((rb["depth"], rb["pixel"]))
    a, b = ra[key_a], rb[key_b]
    assert len(a) == len(b) and len(a) > len(pixels)
    for f in ("pixel", "depth", "flags", "inst", "tri"):
        assert np.array_equal(a[f], b[f]), f
    for f in ("t", "o", "d", "bary", "tp", "light"):
        assert np.array_equal(a[f].view(np.uint32), b[f].view(np.uint32)), f
    ours.close()
    ref.close()


def test_converged_cornell_vs_reference_default_build(ctx, refgpu, cornell_path, halton_perm):
    ours, ref = _pair(ctx, refgpu, cornell_path, halton_perm, 256, 256, exact=False)
    ref.set_settings(spp=16, ray_depth=8)
    a, _ = ours.render(Y.default_setting(spp=16, ray_depth=8), 1)
    b = ref.render_frame(1)
    rmse = float(np.sqrt(np.mean((a[..., :3] - b[..., :3]) ** 2)))
    assert rmse <= 1e-3, rmse
    ours.close()
    ref.close()


@pytest.mark.parametrize("sampler_type", [0, 2])
def test_pcg_and_sobol_vs_reference_cuda(ctx, refgpu, cornell_path, halton_perm, sampler_type):
    ours, ref = _pair(ctx, refgpu, cornell_path, halton_perm, 256, 256, exact=True)
    if sampler_type == 2:
        ours.set_sobol_matrices(refgpu.sobol_matrices())
    ref.set_settings(spp=1, ray_depth=8, sampler_type=sampler_type)
    s = Y.default_setting(spp=1, ray_depth=8, sampler_type=sampler_type)
    a, _ = ours.render(s, 2)
    b = ref.render_frame(2)
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_device_build(f"refcuda_sampler{sampler_type}", ours, ref, s, 2, a, b)
    ours.close()
    ref.close()
