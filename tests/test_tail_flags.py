"""The tables' tail flags (HostKernels::density_tail0 / force_tail0), restated on the CPU.

The density lookups drop the cutoff's select when the W table's last entry (slot 1000) is +0
and every squared distance from cut2 up takes that slot; the force pass's spiky lookup does the
same when that table's last entry is a zero and every distance from h up takes slot 1000. The
flags are computed when the tables are built and choose a template instance of the neighbour
build and of the persistent loop. This restates the host's table build in float32 (the same
operations, correctly rounded division and square root, as HostKernels::build) and checks:
- for the parity scenes (the fuzz generator's 40 parameter sets), both values of each flag
  occur, so the GPU parity suite runs both instances; the wave breaker takes the fast one;
- wherever a flag holds, a squared distance (or distance) at or beyond the cutoff gets slot
  1000 from the device's slot rule and reads a zero there, the value the select gives.
"""
import numpy as np
import pytest

from fuzz_scenes import random_scene
from liquidsimulation_b200 import scenes

f32 = np.float32
K = 1000   # the tables' last slot


def _bits(x):
    return int(np.array([x], np.float32).view(np.uint32)[0])


def _from_bits(b):
    return np.array([b], np.uint32).view(np.float32)[0]


def _smallest(pred, hi):
    """Smallest non-negative float x <= hi with pred(x) (pred monotone), by bisection on bits."""
    lo, top = 0, _bits(hi)
    while lo < top:
        mid = (lo + top) // 2
        if pred(_from_bits(mid)):
            top = mid
        else:
            lo = mid + 1
    return _from_bits(lo)


def tables_tail(radius, factor):
    h = f32(f32(factor) * f32(radius))
    step = f32(h / f32(K))
    r2 = f32(h * h)
    r3 = f32(r2 * h)
    r5 = f32(f32(r3 * h) * h)
    r6 = f32(r5 * h)
    r9 = f32(r6 * r3)
    poly_k = f32(315.0 / (64.0 * np.pi * float(r9)))
    spiky_d1 = f32(-45.0 / (np.pi * float(r6)))
    d = f32(f32(K) * step)
    t = f32(r2 - f32(d * d))
    w_last = f32(f32(f32(poly_k * t) * t) * t)
    s_last = f32(h - d)
    sdw_last = f32(f32(spiky_d1 * s_last) * s_last)
    thr_k = _smallest(lambda x: int(f32(x / step)) >= K, f32(2.0 * h))
    thr2_k = _smallest(lambda s: f32(np.sqrt(f32(s))) >= thr_k, f32(4.0 * h * h + 1.0))
    cut2 = _smallest(lambda s: f32(np.sqrt(f32(s))) >= h, f32(4.0 * h * h + 1.0))
    density = _bits(w_last) == 0 and thr2_k <= cut2
    force = (_bits(sdw_last) & 0x7FFFFFFF) == 0 and thr_k <= h
    return dict(h=h, step=step, thr_k=thr_k, thr2_k=thr2_k, cut2=cut2, w_last=w_last, sdw_last=sdw_last,
                density=density, force=force)


def _slot_guess(d, inv_step):
    # lsp_device.cuh slot_guess: round to nearest of d / step, clamped to [1, 1000]
    k = int(np.rint(np.float64(f32(d * inv_step))))
    return min(max(k, 1), K)


def test_parity_scenes_cover_both_instances():
    flags = [tables_tail(random_scene(k)[0].params.particle_radius, random_scene(k)[0].params.kernel_radius_factor)
             for k in range(40)]
    dens = [f["density"] for f in flags]
    force = [f["force"] for f in flags]
    assert any(dens) and not all(dens)
    assert any(force) and not all(force)
    wb = scenes.wave_breaker(seed=3).params
    f = tables_tail(wb.particle_radius, wb.kernel_radius_factor)
    assert f["density"] and f["force"]


@pytest.mark.parametrize("seed", range(0, 40, 3))
def test_flag_means_the_last_slot_gives_the_cutoff(seed):
    p = random_scene(seed)[0].params
    f = tables_tail(p.particle_radius, p.kernel_radius_factor)
    inv_step = f32(f32(1.0) / f["step"])
    rng = np.random.default_rng(seed)
    if f["density"]:
        # squared distances from cut2 up (the first ones above it, and far beyond)
        c = _bits(f["cut2"])
        for s in [_from_bits(c + k) for k in range(64)] + list(f32(f["cut2"]) * rng.uniform(1.0, 50.0, 64).astype(np.float32)):
            s = f32(s)
            g = f32(np.sqrt(s))   # the device guesses from an approximate root; any root this close gives the same slot
            k = _slot_guess(g, inv_step)
            assert k == K, (s, k)
            assert s >= f["thr2_k"] and _bits(f["w_last"]) == 0
    if f["force"]:
        hb = _bits(f["h"])
        for d in [_from_bits(hb + k) for k in range(64)] + list(f["h"] * rng.uniform(1.0, 7.0, 64).astype(np.float32)):
            d = f32(d)
            assert _slot_guess(d, inv_step) == K and d >= f["thr_k"]
            assert (_bits(f["sdw_last"]) & 0x7FFFFFFF) == 0
