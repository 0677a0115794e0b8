"""FP32 BSDF (eval_surface / pdf_surface, shader.wgsl:1831-2047) against a float64 restatement
over the configurations' whole material ranges, stratified by roughness and by the smaller of
the two cosines.

Materials are drawn the way the flagship configuration draws them (every Disney parameter
uniform over its range: metallic, roughness, specular tint, sheen, sheen tint, clearcoat,
clearcoat gloss, transmission, subsurface in [0, 1]; ior in [1, 2.5]; clearcoat ior in [1, 2])
plus the small configuration's GGX metals (metallic 1, roughness in [0.05, 0.6]).  Half of the
direction pairs are uniform on the sphere (V above the surface); the other half put L near the
mirror direction of V (the normal tilted by a Gaussian of width alpha), where the GGX lobe
peaks.  The relative error of a sample is
max_c |f32_c - f64_c| / max_c |f64_c| for the value and |pdf32 - pdf64| / pdf64 for the pdf.

The 1e-5 bar holds where the GGX lobe is well conditioned (roughness >= 0.3, both cosines >=
0.2).  Near the peaks (alpha^2 clamped at 1e-6, so D reaches 1e5 and FP32 loses digits in
1 + (alpha^2 - 1) cos^2) and at grazing angles it does not, in either implementation of the
same formula; those strata are measured and reported, not excluded.  `python
tests/test_bsdf_strata.py` prints the table.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import host_oracle as ho
from webgpuraytracer_b200 import scene as sc

ROUGH_BINS = [(0.0, 0.1), (0.1, 0.3), (0.3, 0.6), (0.6, 1.0001)]
COS_BINS = [(0.0, 0.05), (0.05, 0.2), (0.2, 1.0001)]
KINDS = ("uniform", "near the mirror direction")
N_MATERIALS = 96
PAIRS_PER_MATERIAL = 128


def _draw_material(rng, metal: bool):
    u = lambda lo=0.0, hi=1.0: float(rng.uniform(lo, hi))
    if metal:
        return sc.Material("m", [u(0.1, 0.9) for _ in range(3)], u(0.05, 0.6), metallic=1.0)
    return sc.Material("d", [u(0.1, 0.9) for _ in range(3)], u(), metallic=u(), ior=u(1.0, 2.5),
                       specularTint=u(), anisotropic=u(), anisotropicRotation=u(), sheen=u(), sheenTint=u(),
                       clearcoat=u(), clearcoatGloss=u(), clearcoatIor=u(1.0, 2.0), transmission=u(),
                       subsurface=u(), concentration=u(0.0, 2.0))


def strata(seed: int = 7):
    """{(kind, rough_bin, cos_bin): (value rel errors, pdf rel errors)} over the drawn samples."""
    rng = np.random.default_rng(seed)
    out = {(k, i, j): ([], []) for k in range(len(KINDS)) for i in range(len(ROUGH_BINS))
           for j in range(len(COS_BINS))}
    n = [0.0, 0.0, 1.0]
    for k in range(N_MATERIALS):
        mat = _draw_material(rng, metal=(k % 4 == 3))
        mat._index = 0
        buf, _ = sc.pack_data_from_schema([mat], lambda x: x.schema(), sc._MAT_EMPTY)
        buf = np.ascontiguousarray(buf[:144])
        f32 = buf.view(np.float32)
        albedo = f32[0:3]
        rough, metal = float(f32[4]), float(f32[3])
        mref = {"subsurface_tint": f32[16:19].astype(np.float64)}
        for i, key in ((5, "ior"), (6, "specular_tint"), (9, "sheen"), (10, "sheen_tint"), (11, "clearcoat"),
                       (12, "clearcoat_gloss"), (13, "clearcoat_ior"), (14, "transmission"), (19, "subsurface")):
            mref[key] = float(f32[i])
        vl = rng.normal(size=(PAIRS_PER_MATERIAL, 6))
        vl[:, :3] /= np.linalg.norm(vl[:, :3], axis=1, keepdims=True)
        vl[:, 3:] /= np.linalg.norm(vl[:, 3:], axis=1, keepdims=True)
        vl[:, 2] = np.abs(vl[:, 2])
        half = PAIRS_PER_MATERIAL // 2
        alpha = max(rough, 0.01) ** 2
        for s in range(half, PAIRS_PER_MATERIAL):     # L near the mirror direction of V
            h = np.array([0.0, 0.0, 1.0]) + np.append(rng.normal(scale=alpha, size=2), 0.0)
            h /= np.linalg.norm(h)
            V = vl[s, :3]
            vl[s, 3:] = -V + 2 * np.dot(V, h) * h
        vl = vl.astype(np.float32)
        f, pdf = oracle.bsdf(buf, n, rough, metal, albedo, vl)
        rb = next(i for i, (lo, hi) in enumerate(ROUGH_BINS) if lo <= rough < hi)
        for s in range(len(vl)):
            fr, pr = ho.bsdf_f64(mref, n, albedo.astype(np.float64), rough, metal, vl[s, :3].astype(np.float64),
                                 vl[s, 3:].astype(np.float64))
            mag = float(np.max(np.abs(fr)))
            if mag == 0.0 and pr <= 1e-7:
                continue                      # both report "no contribution"
            c = min(abs(float(vl[s, 2])), abs(float(vl[s, 5])))
            cb = next(j for j, (lo, hi) in enumerate(COS_BINS) if lo <= c < hi)
            ev = float(np.max(np.abs(f[s] - fr))) / mag if mag > 0 else float(np.max(np.abs(f[s])) > 0)
            ep = abs(float(pdf[s]) - pr) / pr
            kind = 0 if s < half else 1
            out[(kind, rb, cb)][0].append(ev)
            out[(kind, rb, cb)][1].append(ep)
    return out


def table(st) -> list[dict]:
    rows = []
    for (k, i, j), (ev, ep) in sorted(st.items()):
        ev, ep = np.array(ev), np.array(ep)
        rows.append({"directions": KINDS[k], "roughness": ROUGH_BINS[i], "min_cos": COS_BINS[j],
                     "samples": int(ev.size),
                     "value_within_1e-5": float(np.mean(ev <= 1e-5)) if ev.size else None,
                     "pdf_within_1e-5": float(np.mean(ep <= 1e-5)) if ep.size else None,
                     "value_p99": float(np.quantile(ev, 0.99)) if ev.size else None,
                     "pdf_p99": float(np.quantile(ep, 0.99)) if ep.size else None})
    return rows


@pytest.fixture(scope="module")
def rows():
    return table(strata())


def test_well_conditioned_strata_meet_1e5(rows):
    for r in rows:
        if r["directions"] == KINDS[0] and r["roughness"][0] >= 0.3 and r["min_cos"][0] >= 0.2:
            assert r["samples"] >= 100
            assert r["value_within_1e-5"] >= 0.99, r
            assert r["pdf_within_1e-5"] >= 0.99, r


def test_every_stratum_is_measured_and_bounded(rows):
    """Each stratum has samples, and 99 % of its FP32 results stay within the error the FP32
    evaluation of the same formula can reach: 1e-2 everywhere except at the peak of the sharpest
    lobes (roughness < 0.1, alpha^2 at its 1e-6 clamp), where 1 - cos^2 (of order alpha^2)
    is formed from cos^2 = 1 - O(1e-6) with an FP32 rounding error of 6e-8, a relative error of
    ~6e-2 that D squares; there the bound is 0.1."""
    for r in rows:
        bound = 0.1 if (r["directions"] == KINDS[1] and r["roughness"][1] <= 0.1) else 1e-2
        assert r["samples"] >= 20, r
        assert r["value_p99"] <= bound, r
        assert r["pdf_p99"] <= bound, r


if __name__ == "__main__":
    print("| directions | roughness | min cos | samples | value within 1e-5 | pdf within 1e-5 | value p99 rel err | "
          "pdf p99 rel err |")
    print("|---|---|---|---|---|---|---|---|")
    for r in table(strata()):
        print(f"| {r['directions']} | {r['roughness'][0]:.1f}-{min(r['roughness'][1], 1.0):.1f} | {r['min_cos'][0]:.2f}-"
              f"{min(r['min_cos'][1], 1.0):.2f} | {r['samples']} | {r['value_within_1e-5']:.3f} | "
              f"{r['pdf_within_1e-5']:.3f} | {r['value_p99']:.1e} | {r['pdf_p99']:.1e} |")
