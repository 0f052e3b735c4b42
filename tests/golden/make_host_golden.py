"""Writes tests/golden/host_golden.npz: golden vectors for the host-side
logic of the search path, taken from the reference itself.

  * the acceleration list of the reference's example run, parsed from its
    shipped example_output/overview.xml (10,758 trials at DM 54.5);
  * acceleration lists produced by the reference's own AccelerationPlan
    (include/utils/utils.hpp) built from its sources (oracle/_ref), for a
    grid of DMs and the configurations of the benchmark workloads;
  * outputs of the reference's own HarmonicDistiller, AccelerationDistiller
    and DMDistiller (include/transforms/distiller.hpp) on seeded synthetic
    candidate lists.

Run here, where the reference sources exist:
    python tests/golden/make_host_golden.py [reference_root]
"""
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402


def overview_accels(ref_root):
    txt = open(os.path.join(ref_root, "example_output", "overview.xml")).read()
    blk = txt[txt.index("<acceleration_trials"):txt.index("</acceleration_trials>")]
    vals = re.findall(r"<trial id='\d+'>([^<]+)</trial>", blk)
    return np.array([float(v) for v in vals], np.float32)


def cand_list(rng, n, nh_max=5):
    f0 = rng.uniform(0.5, 200.0, size=max(1, n // 4))
    out = np.zeros(n, O.CAND_DTYPE)
    for i in range(n):
        base = f0[rng.integers(f0.size)]
        h = rng.integers(1, 17)
        k = 2 ** rng.integers(0, nh_max + 1)
        freq = base * h / k * (1 + rng.normal(0, 3e-5)) if rng.uniform() < 0.7 else rng.uniform(0.1, 1000)
        out[i] = (10.0, 3, rng.choice([-50.0, -10.0, 0.0, 10.0, 50.0]), rng.integers(0, nh_max + 1),
                  np.float32(rng.uniform(6, 40)), np.float32(freq))
    # a few exact S/N ties
    out["snr"][1::17] = out["snr"][0::17][:len(out["snr"][1::17])]
    return out


def main(ref_root="/root/reference"):
    O.build_reference(ref_root)
    g = {}
    g["overview_accels"] = overview_accels(ref_root)
    # example run parameters (overview.xml <header_parameters>, <search_parameters>)
    fch1, foff, nch = 1079.43359375, -8.5, 64
    cf = np.float32(fch1 + foff * nch / 2)
    ov = (-150.0, 150.0, float(np.float32(1.11)), 64e-6, 1 << 28, float(np.float32(1.5058824e-05)),
          float(np.float32(np.float64(cf) * 1e6)), float(np.float32(np.float64(np.float32(foff)) * 1e6)))
    g["overview_args"] = np.array(ov[:4] + ov[5:], np.float64)
    g["overview_nsamps"] = np.int64(ov[4])
    from peasoup_b200 import synth
    cases = []
    # (acc_lo, acc_hi, tol, pw, nsamps, tsamp, cfreq, chbw, cdm)
    cases.append((-50.0, 50.0, 1.10, 64e-6, 1 << 20, 64e-6, synth.CFREQ_HZ, synth.CH_BW_HZ, 0.0))
    cases.append((-100.0, 100.0, 1.10, 64e-6, 1 << 23, 76e-6, synth.CFREQ_HZ, synth.CH_BW_HZ, 0.0))
    cases.append((-50.0, 50.0, 1.10, 64e-6, 1 << 22, 64e-6, synth.CFREQ_HZ, synth.CH_BW_HZ, 0.0))
    cases.append((-500.0, 500.0, 1.10, 64e-6, 1 << 27, 64e-6, synth.CFREQ_HZ, synth.CH_BW_HZ, 0.0))
    cases.append((-300.0, 10.0, 1.10, 64e-6, 3 << 20, 64e-6, synth.CFREQ_HZ, synth.CH_BW_HZ, 30.0))
    cases.append(ov + (54.5,))
    dms = np.array([0.0, 0.5, 7.5, 30.0, 54.5, 127.5, 500.0], np.float32)
    lists, index, offset = [], [], 0
    for ci, c in enumerate(cases):
        # the long cases (10^4-10^5 trials per DM) at two DMs only
        for dm in (dms if ci not in (3, 5) else np.array([c[8], 127.5], np.float32)):
            a = O.ref_accel_list(*[float(v) if not isinstance(v, int) else v for v in c[:8]],
                                 float(dm), float(c[8]))
            index.append((ci, float(dm), offset, a.size))
            lists.append(a)
            offset += a.size
    g["accel_cases"] = np.array([list(c[:4]) + [float(c[4])] + list(c[5:]) for c in cases], np.float64)
    g["accel_dms"] = dms
    g["accel_index"] = np.array(index, np.float64)
    g["accel_values"] = np.concatenate(lists).astype(np.float32)
    rng = np.random.default_rng(7)
    for name, kind, kw in (("harm", 0, dict(tol=1e-4, max_harm=16.0, keep_related=False, fractional=True)),
                           ("harm_related", 0, dict(tol=1e-4, max_harm=16.0, keep_related=True, fractional=False)),
                           ("accel", 1, dict(tol=1e-4, tobs=637.5, keep_related=True)),
                           ("dm", 2, dict(tol=1e-4, keep_related=True))):
        for j, n in enumerate((1, 7, 60, 300)):
            c = cand_list(rng, n)
            out, na = O.ref_distill(kind, c, **kw)
            g[f"distill_{name}_{j}_in"] = c
            g[f"distill_{name}_{j}_out"] = out
            g[f"distill_{name}_{j}_nassoc"] = na
    path = os.path.join(ROOT, "tests", "golden", "host_golden.npz")
    np.savez_compressed(path, **g)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(*sys.argv[1:])
