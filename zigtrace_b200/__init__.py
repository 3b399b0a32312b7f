"""zigtrace_b200 -- B200-native (sm_100a) renderer for zigtrace's per-pixel
radiance path, behind a mirror of the reference library API.

    import zigtrace_b200 as zt
    scene = zt.Scene()
    white = scene.add_material(zt.Material.lambertian((0.73, 0.73, 0.73)))
    scene.add_quad((0, 0, 0), (555, 0, 0), (0, 0, 555), white)
    scene.build()
    img = zt.render(scene, zt.Options(width=256, height=256, spp=64, max_depth=16))
    rgb = img.to_rgb8(zt.Output(tonemap="aces"))
"""
from .api import (  # noqa: F401
    DIELECTRIC, EMISSIVE, LAMBERTIAN, METAL, MODE_AUTO, MODE_MEGAKERNEL, MODE_MEGAKERNEL_REGEN, MODE_WAVEFRONT, MODE_WAVEFRONT_SORTED, PLANE, PRECISION_EXACT, PRECISION_FAST, SPHERE, TRIANGLE,
    Background, Batch, CameraConfig, GpuConfig, Image, Material, Options, Output, Scene, Settings, ZigtraceError,
    backward, backward_rows, encode_png, encode_png_device, forward, forward_rows, image_to_rgb8_device, plane, png_size, render, render_batch,
    render_debug, render_device, render_function, render_rows_device, render_png, render_rgb8, rng_streams, set_colors, sphere, triangle,
    write_png, write_ppm)

__version__ = "0.1.0"
