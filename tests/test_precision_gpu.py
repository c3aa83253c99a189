"""Precision variants on the Weibel set-up (128x128 cells, two species, 4x4
ppc, ThermalCorr uth 0.1, uz +-0.6; openmp/em2d/main.cpp:179-259), compared
with the FP64 restatement of the same step at steps 100 and 500:

* the CUDA step in FP32 (the reference's arithmetic) with the tile current
  summed by FP32 shared atomics (option "jacc" 0), by FP64 atomics ("jacc"
  1) and in fixed point (the default, "jacc" 2),
* the FP32 oracle (the reference's scalar FP32 build, restated),
* the FP32 oracle with the momenta rounded to BF16 after every step -- the
  storage format a BF16-momentum variant would use (BF16 carries its own
  exponent, so a per-species scale changes nothing here).

All runs start from the same FP32 initial state.  The figures are written as
JSON to the file named by ZPIC_PRECISION_OUT when that variable is set."""
import json
import os

import numpy as np
import pytest

from em2d_oracle import OracleSim, weibel_setup
import zpic_b200 as zb

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

GEOM = ((8, 8), (16, 16), (12.8, 12.8), 0.07)
CHECKS = (100, 500)


def to_bf16(a):
    """Round FP32 values to BF16 (round to nearest even) and widen back."""
    b = np.ascontiguousarray(a, np.float32).view(np.uint32)
    r = ((b >> 16) & 1) + np.uint32(0x7FFF)
    return ((b + r) & np.uint32(0xFFFF0000)).view(np.float32)


def energies(s):
    e, b = s.emf_energy()
    return float(e.sum() + b.sum()), s.species_energy(0) + s.species_energy(1)


def copy_state(src, dst, cast=None):
    for sp in range(2):
        npt, ix, x, u = src.particles(sp)
        if cast is not None:
            u = cast(u)
        dst.set_particles(sp, npt, ix, x, u)


def run_history(sim, per_step=None):
    out = {}
    n = 0
    for target in CHECKS:
        while n < target:
            if per_step is None:
                sim.advance(target - n)
                n = target
            else:
                sim.advance(1)
                per_step(sim)
                n += 1
        out[target] = energies(sim)
    return out


def test_precision_variants_against_fp64():
    o32 = weibel_setup(OracleSim(*GEOM, real='f32'))
    o64 = weibel_setup(OracleSim(*GEOM, real='f64'))
    obf = weibel_setup(OracleSim(*GEOM, real='f32'))
    g32 = weibel_setup(zb.Simulation(*GEOM))
    g32.set_option('jacc', 0)
    gj = weibel_setup(zb.Simulation(*GEOM))
    gj.set_option('jacc', 1)
    gx = weibel_setup(zb.Simulation(*GEOM))
    gx.set_option('jacc', 2)
    copy_state(o32, o64)
    copy_state(o32, obf, to_bf16)
    copy_state(o32, g32)
    copy_state(o32, gj)
    copy_state(o32, gx)

    def bf16_round(s):
        copy_state(s, s, to_bf16)

    hist = {
        'fp64 oracle': run_history(o64),
        'fp32 oracle': run_history(o32),
        'cuda fp32, fp32 tile current': run_history(g32),
        'cuda fp32, fp64 tile current': run_history(gj),
        'cuda fp32, fixed-point tile current': run_history(gx),
        'fp32 oracle, bf16 momenta': run_history(obf, bf16_round),
    }
    ref = hist['fp64 oracle']
    report = {}
    for name, h in hist.items():
        report[name] = {}
        for n in CHECKS:
            fe, ke = h[n]
            report[name][n] = {
                'field_energy': fe, 'kinetic_energy': ke,
                'field_rel_err': abs(fe - ref[n][0]) / ref[n][0],
                'kinetic_rel_err': abs(ke - ref[n][1]) / ref[n][1],
            }
    path = os.environ.get('ZPIC_PRECISION_OUT')
    if path:
        with open(path, 'w') as f:
            json.dump(report, f, indent=1)
    for name in ('fp32 oracle', 'cuda fp32, fp32 tile current', 'cuda fp32, fp64 tile current',
                 'cuda fp32, fixed-point tile current'):
        r = report[name]
        # FP32 round-off against FP64 before and after the Weibel saturation:
        # field and kinetic energy within 1e-4 of the FP64 path at step 500
        for n in CHECKS:
            assert r[n]['kinetic_rel_err'] < 1e-4, (name, n, r)
            assert r[n]['field_rel_err'] < 1e-4, (name, n, r)
    for n in CHECKS:
        assert np.isfinite(report['fp32 oracle, bf16 momenta'][n]['field_energy'])
