"""Algorithmic work per sample, for the roofline.

The renderer is neither a dense contraction nor a streaming kernel: its time
goes to f64 arithmetic in BVH traversal and shading, and to dependent loads
of BVH records.  Work is counted per sample by the instrumented oracle on the
same workload (counts of box tests, primitive tests, hits and light samples),
then converted with fixed per-operation costs counted from the reference's
arithmetic (f64 add/sub/mul/div/sqrt, no FMA in the renderer; compares not
counted):

  box slab test       12  (aabb.zig:74-75: 2 sub + 2 mul per axis)
  sphere test         26  (geometry.zig:38-45)
  triangle test       52  (geometry.zig:84-96, with the two edge subtractions)
  plane test          14  (geometry.zig:68-70)
  shading per hit     60  (hit record, emission, scatter, roulette)
  light sample        50  (light.zig:120-166 and render.zig:46-56 minus the shadow ray)

Bytes per sample count what one traversal step reads in the device layout:
128 B per interior-node visit (one DPair record), 80 B per primitive test
(one DPrim record), plus the 24-byte f64 pixel written once per pixel.
"""
from __future__ import annotations

FLOP_SLAB = 12
FLOP_SPHERE = 26
FLOP_TRIANGLE = 52
FLOP_PLANE = 14
FLOP_SHADE = 60
FLOP_NEE = 50
BYTES_PAIR = 128
BYTES_PRIM = 80
BYTES_PIXEL = 24


BYTES_FPAIR = 64  # the fast traversal's single-precision pair record


def per_sample(stats: dict, spp: int, has_bvh: bool = True, fast: bool = False) -> dict:
    """Per-sample FLOP and bytes from oracle counters (oracle.STATS_FIELDS).
    With fast=True (the fast traversal) the box tests are single-precision
    FMAs on 64-byte records: their FLOP are reported apart as flop_f32 and
    the node records count 64 bytes."""
    n = max(stats["samples"], 1)
    traversals = (stats["ext_rays"] + stats["shadow_rays"]) if has_bvh else 0
    inner_pops = max(stats["slab_tests"] - traversals, 0) / 2
    prim_tests = stats["sphere_tests"] + stats["tri_tests"] + stats["plane_tests"]
    flop = (FLOP_SLAB * stats["slab_tests"] + FLOP_SPHERE * stats["sphere_tests"] +
            FLOP_TRIANGLE * stats["tri_tests"] + FLOP_PLANE * stats["plane_tests"] + FLOP_SHADE * stats["hits"] +
            FLOP_NEE * stats["nee_samples"]) / n
    nbytes = ((BYTES_FPAIR if fast else BYTES_PAIR) * inner_pops + BYTES_PRIM * prim_tests) / n + BYTES_PIXEL / spp
    flop_f32 = FLOP_SLAB * stats["slab_tests"] / n if fast else 0.0
    return {
        "flop": flop,
        "flop_f32": flop_f32,
        "bytes": nbytes,
        "ext_rays": stats["ext_rays"] / n,
        "shadow_rays": stats["shadow_rays"] / n,
        "box_tests": stats["slab_tests"] / n,
        "prim_tests": prim_tests / n,
    }


# Path-state bytes the wavefront form moves through HBM (wavefront.cuh's
# WfState, f64 SoA), counted from its kernels:
#   per sample   start + finish: ray, throughput, radiance, previous hit,
#                depth, flags, RNG state, sample index, pixel sum, queue push
#   per ray      k_wf_extend (queue index, ray in; hit t and id out) and the
#                part of k_wf_shade every ray pays (RNG, ray, throughput,
#                radiance, hit id in; radiance and RNG out)
#   per hit      hit t, depth; the scattered ray, throughput, previous hit,
#                depth and queue push written back
#   per shadow   the light sample written by k_wf_shade (13 doubles + push)
#                and k_wf_shadow's reads, radiance update and flags
WF_BYTES_SAMPLE = 256
WF_BYTES_RAY = 64 + 136 + 56
WF_BYTES_HIT = 8 + 4 + 116
WF_BYTES_SHADOW = 108 + 160


def wavefront_queue_bytes(stats: dict, spp: int) -> float:
    """Path-state bytes per sample of the wavefront form, from oracle counters."""
    n = max(stats["samples"], 1)
    return (WF_BYTES_SAMPLE + (WF_BYTES_RAY * stats["ext_rays"] + WF_BYTES_HIT * stats["hits"] +
                               WF_BYTES_SHADOW * stats["shadow_rays"]) / n + BYTES_PIXEL / spp)
