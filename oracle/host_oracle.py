"""ORACLE -- test infrastructure only.  Python restatements of tracer.js's host-side builders,
used to check the native builders of libwgpt.so on small inputs.

    blas_build    ModelData.generateBVH (tracer.js:1025-1118), binned SAH, DFS flatten
    tlas_build    SceneBVHBuilder.recursiveBuild + flatten (tracer.js:1533-1619)
    env_cdf       HDRTexture.buildHDRCDF (tracer.js:135-204)
    decode_rgbe   parseHdr (lib/parse-hdr.js:20-211) + HDRTexture.updateData (tracer.js:76-87)
    bsdf_f64      eval_surface / pdf_surface (shader.wgsl:1831-2047) in float64, the reference for
                  the single-precision BSDF's error bound

JavaScript numbers are doubles: Python floats reproduce them exactly; Float32Array /
Float16Array stores are numpy float32 / float16 conversions (round to nearest even).
"""
from __future__ import annotations

import math

import numpy as np


def _f32(x) -> float:
    return float(np.float32(x))


# ----------------------------------------------------------------------------- BLAS
def blas_build(tris24: np.ndarray):
    """Returns (nodes as a list of (min3, max3, num, next), flat triangle order as indices)."""
    t = np.asarray(tris24, dtype=np.float32).reshape(-1, 24)
    n = len(t)
    verts = [[[float(t[i, v * 3 + k]) for k in range(3)] for v in range(3)] for i in range(n)]
    cent = [[(verts[i][0][k] + verts[i][1][k] + verts[i][2][k]) / 3 for k in range(3)] for i in range(n)]

    def bounds(idx):
        mn = [math.inf] * 3
        mx = [-math.inf] * 3
        for i in idx:
            for v in verts[i]:
                for k in range(3):
                    mn[k] = min(mn[k], v[k])
                    mx[k] = max(mx[k], v[k])
        return mn, mx

    def area(mn, mx):
        d = [mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]]
        return 2 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0])

    def subdivide(idx):
        mn, mx = bounds(idx)
        best_cost = len(idx) * area(mn, mx)
        best_axis, best_split = -1, -1
        for axis in range(3):
            start, end = mn[axis], mx[axis]
            if end - start < 1e-6:
                continue
            num_bins = min(len(idx), 12)
            for i in range(1, num_bins):
                split = start + (i / num_bins) * (end - start)
                left = [j for j in idx if cent[j][axis] < split]
                right = [j for j in idx if not cent[j][axis] < split]
                if not left or not right:
                    continue
                bl, br = bounds(left), bounds(right)
                cost = len(left) * area(*bl) + len(right) * area(*br)
                if cost < best_cost:
                    best_cost, best_axis, best_split = cost, axis, split
        if best_axis == -1 or len(idx) <= 2:
            return {"min": mn, "max": mx, "indices": idx}
        left = [j for j in idx if cent[j][best_axis] < best_split]
        right = [j for j in idx if not cent[j][best_axis] < best_split]
        return {"min": mn, "max": mx, "left": subdivide(left), "right": subdivide(right)}

    root = subdivide(list(range(n)))
    nodes, flat = [], []

    def flatten(node):
        index = len(nodes)
        rec = [node["min"], node["max"], 0, 0]
        nodes.append(rec)
        if "indices" in node:
            rec[2] = len(node["indices"])
            rec[3] = len(flat)
            flat.extend(node["indices"])
        else:
            flatten(node["left"])
            rec[3] = flatten(node["right"])
        return index

    flatten(root)
    return nodes, flat


def nodes_to_bytes(nodes) -> np.ndarray:
    out = np.zeros((len(nodes), 8), dtype=np.uint32)
    f = out.view(np.float32)
    for i, (mn, mx, num, nxt) in enumerate(nodes):
        f[i, 0:3] = np.float32(mn)
        f[i, 4:7] = np.float32(mx)
        out[i, 3] = num
        out[i, 7] = nxt
    return out.view(np.uint8).reshape(-1)


# ----------------------------------------------------------------------------- TLAS
def tlas_build(aabbs: np.ndarray) -> np.ndarray:
    """aabbs: n x 6 float32 (min, max) -> flattened nodes (bytes)."""
    a = np.asarray(aabbs, dtype=np.float32).reshape(-1, 6)
    items = [{"index": i, "min": [float(v) for v in a[i, :3]], "max": [float(v) for v in a[i, 3:]]}
             for i in range(len(a))]
    nodes = []

    def build(its, depth):
        node = {"min": None, "max": None, "num": 0, "obj": -1, "next": -1}
        nodes.append(node)
        mn = [math.inf] * 3
        mx = [-math.inf] * 3
        for it in its:
            for k in range(3):
                mn[k] = _f32(min(mn[k], it["min"][k]))
                mx[k] = _f32(max(mx[k], it["max"][k]))
        node["min"], node["max"] = mn, mx
        if len(its) <= 1 or depth > 20:
            node["num"] = len(its)
            node["obj"] = its[0]["index"]
            return
        size = [_f32(mx[k] - mn[k]) for k in range(3)]
        axis = 0
        if size[1] > size[0]:
            axis = 1
        if size[2] > size[axis]:
            axis = 2
        its = sorted(its, key=lambda it: (it["min"][axis] + it["max"][axis]) * 0.5)   # stable, like V8
        mid = len(its) // 2
        build(its[:mid], depth + 1)
        node["next"] = len(nodes)
        build(its[mid:], depth + 1)

    if len(items):
        build(items, 0)
    recs = [(nd["min"], nd["max"], nd["num"], nd["obj"] if nd["num"] > 0 else nd["next"]) for nd in nodes]
    return nodes_to_bytes(recs)


# ----------------------------------------------------------------------------- environment
def env_cdf(data16: np.ndarray, width: int, height: int, exposure: float = 1.0):
    """Returns (float32 CDF buffer, sky_cdf_index, totalWeight)."""
    d = np.asarray(data16, dtype=np.uint16).view(np.float16).astype(np.float64).reshape(height, width, 4)
    thr = 65536 - 16 - 1
    marg = np.zeros(height + 1, dtype=np.float32)
    cond = np.zeros(height * (width + 1), dtype=np.float32)
    total = 0.0
    for y in range(height):
        sin_t = math.sin(math.pi * (y + 0.5) / height)
        r = np.minimum(d[y, :, 0] * exposure, thr)
        g = np.minimum(d[y, :, 1] * exposure, thr)
        b = np.minimum(d[y, :, 2] * exposure, thr)
        lum = (0.2126 * r + 0.7152 * g + 0.0722 * b) * sin_t
        run = np.cumsum(lum)                       # sequential accumulation, as `rowWeight += lum`
        row_w = float(run[-1]) if width else 0.0
        base = y * (width + 1)
        cond[base + 1:base + width + 1] = run.astype(np.float32)
        if row_w > 0:
            cond[base + 1:base + width + 1] = (cond[base + 1:base + width + 1].astype(np.float64) / row_w).astype(np.float32)
        else:
            cond[base + 1:base + width + 1] = (np.arange(1, width + 1) / width).astype(np.float32)
        total += row_w
        marg[y + 1] = np.float32(total)
    if total > 0:
        marg[1:] = (marg[1:].astype(np.float64) / total).astype(np.float32)
    else:
        marg[1:] = (np.arange(1, height + 1) / height).astype(np.float32)
    return np.concatenate([marg, cond]), height + 1, total


def decode_rgbe(buf: bytes, exposure: float = 1.0) -> tuple[np.ndarray, int, int]:
    """Radiance RGBE (run-length encoded) -> (rgba16f as uint16 [h*w*4], w, h)."""
    off = 0
    n = len(buf)

    def read_line():
        nonlocal off
        s = bytearray()
        while off < n:
            b = buf[off]
            off += 1
            if b == 10:
                break
            s.append(b)
        return s.decode("latin-1")

    w = h = 0
    rle = False
    for _ in range(20):
        line = read_line()
        if "#?RADIANCE" in line:
            continue
        if "FORMAT=32-bit_rle_rgbe" in line:
            rle = True
            continue
        if "EXPOSURE=" in line or "#" in line:
            continue
        parts = line.split()
        if len(parts) == 4 and parts[0] == "-Y" and parts[2] == "+X":
            h, w = int(parts[1]), int(parts[3])
            break
    if not rle:
        raise ValueError("File is not run length encoded!")
    data = np.zeros((h, w, 4), dtype=np.uint8)
    for y in range(h):
        hdr = buf[off:off + 4]
        off += 4
        if hdr[0] != 2 or hdr[1] != 2 or (hdr[2] & 0x80):
            flat = np.frombuffer(bytes(hdr) + buf[off:off + (w * (h - y) - 1) * 4], dtype=np.uint8)
            data[y:] = flat.reshape(h - y, w, 4)
            break
        if ((hdr[2] << 8) | hdr[3]) != w:
            raise ValueError("Wrong scanline width")
        for ch in range(4):
            ptr = 0
            while ptr < w:
                b0, b1 = buf[off], buf[off + 1]
                off += 2
                if b0 > 128:
                    cnt = b0 - 128
                    data[y, ptr:ptr + cnt, ch] = b1
                    ptr += cnt
                else:
                    cnt = b0
                    data[y, ptr, ch] = b1
                    ptr += 1
                    if cnt > 1:
                        data[y, ptr:ptr + cnt - 1, ch] = np.frombuffer(buf[off:off + cnt - 1], dtype=np.uint8)
                        ptr += cnt - 1
                        off += cnt - 1
    f = np.ldexp(1.0, data[..., 3].astype(np.int64) - 128)
    rgb = (data[..., :3].astype(np.float64) / 255) * f[..., None]
    rgb32 = rgb.astype(np.float32)                               # Float32Array of parseHdr
    v = np.minimum(rgb32.astype(np.float64) * exposure, 65536 - 16 - 1)
    out = np.ones((h, w, 4), dtype=np.float64)
    out[..., :3] = v
    return out.astype(np.float16).view(np.uint16).reshape(-1), w, h


# ----------------------------------------------------------------------------- BSDF (float64)
def _fresnel_dielectric(c, etai, etat):
    c = min(max(abs(c), 0.0), 1.0)
    sint = (etai / etat) * math.sqrt(max(0.0, 1 - c * c))
    if sint >= 1:
        return 1.0
    cost = math.sqrt(max(0.0, 1 - sint * sint))
    rs = (etat * c - etai * cost) / (etat * c + etai * cost)
    rp = (etai * c - etat * cost) / (etai * c + etat * cost)
    return (rs * rs + rp * rp) / 2


def _D(nh, a2):
    den = nh * nh * (a2 - 1) + 1
    return a2 / (math.pi * den * den + 1e-10)


def _G2(nv, nl, a2):
    sv = math.sqrt(max(0.0, a2 + nv * nv * (1 - a2)))
    sl = math.sqrt(max(0.0, a2 + nl * nl * (1 - a2)))
    return 2 * nl / (nl * sv + nv * sl + 1e-10)


def _G2u(nv, nl, a2):
    lv = nv + math.sqrt(max(0.0, a2 + nv * nv * (1 - a2)))
    ll = nl + math.sqrt(max(0.0, a2 + nl * nl * (1 - a2)))
    return 4 * nl / (lv * ll + 1e-7)


def _G1(nv, a2):
    return 2 / (nv + math.sqrt(max(0.0, a2 + (1 - a2) * nv * nv)) + 1e-7)


def bsdf_f64(mat: dict, normal, albedo, roughness, metallic, V, L):
    """eval_surface and pdf_surface (shader.wgsl:1831-2047) in double precision, air outside
    (empty medium stack), alpha = 1.  mat keys: ior, specular_tint, sheen, sheen_tint,
    subsurface, subsurface_tint, clearcoat, clearcoat_gloss, clearcoat_ior, transmission."""
    n = np.asarray(normal, np.float64)
    V = np.asarray(V, np.float64)
    L = np.asarray(L, np.float64)
    alb = np.asarray(albedo, np.float64)
    entering = float(n @ V) > 0
    no = n if entering else -n
    nv, nl = float(no @ V), float(no @ L)
    if nv <= 0:
        return np.zeros(3), 1e-7
    rv = min(max(roughness, 0.01), 1.0)
    alpha = rv * rv
    a2 = max(alpha * alpha, 1e-6)
    etai, etat = (1.0, mat["ior"]) if entering else (1.0, 1.0)
    trans = mat["transmission"]
    Fcc = _fresnel_dielectric(nv, 1.0, mat["clearcoat_ior"])
    p_cc = mat["clearcoat"] * Fcc if entering else 0.0
    F_est = (1 - rv) * _fresnel_dielectric(nv, etai, etat) + rv * ((etai - etat) / (etai + etat)) ** 2
    pw = max(0.0, 1 - nv) ** 5
    F_metal = alb + (1 - alb) * pw
    F_act = F_est * (1 - metallic) + F_metal * metallic
    f_avg = min(max(float(F_act.sum()) / 3, 0.0), 1.0)
    p_spec = (1 - p_cc) * f_avg
    p_trans = (1 - p_cc) * (1 - f_avg) * trans * (1 - metallic)
    p_diff = (1 - p_cc) * (1 - f_avg) * (1 - trans) * (1 - metallic)
    f = np.zeros(3)
    pdf = 0.0
    cc_r = min(max(1 - mat["clearcoat_gloss"], 0.01), 1.0)
    cc_a2 = max((cc_r * cc_r) ** 2, 1e-6)
    if nl > 0:
        Hv = V + L
        H = Hv / np.linalg.norm(Hv) if float(Hv @ Hv) > 1e-6 else no
        nh = max(float(no @ H), 0.0)
        vh = max(float(V @ H), 0.0)
        D = _D(nh, a2)
        dc = alb.copy()
        if mat["sheen"] > 0:
            dc = dc + (1 * (1 - mat["sheen_tint"]) + alb * mat["sheen_tint"]) * pw * mat["sheen"]
        if mat["subsurface"] > 0:
            dc = dc * (1 - mat["subsurface"]) + np.asarray(mat["subsurface_tint"]) * mat["subsurface"]
        diffuse = dc / math.pi * (1 - metallic) * (1 - trans)
        Fd = _fresnel_dielectric(vh, etai, etat)
        lum = float(alb @ np.array([0.2126, 0.7152, 0.0722]))
        tint = np.ones(3) if lum <= 0 else alb / max(lum, 1e-4)
        st = mat["specular_tint"]
        Fdt = Fd * (1 - st) + Fd * tint * st
        F90 = (1 - st) + tint * st
        Fm = alb + (F90 - alb) * max(0.0, 1 - vh) ** 5
        Fa = Fdt * (1 - metallic) + Fm * metallic
        diffuse_cos = diffuse * nl * (1 - F_act)
        spec = D * Fa * _G2(nv, nl, a2) / 4 * (1 + alpha * 0.4)
        cc_cos = np.zeros(3)
        cc_att = 1.0
        if mat["clearcoat"] > 0 and entering:
            cc_cos = np.full(3, mat["clearcoat"] * _D(nh, cc_a2) * _G2(nv, nl, cc_a2)
                             * _fresnel_dielectric(vh, 1.0, mat["clearcoat_ior"]) / 4)
            cc_att = 1 - mat["clearcoat"] * Fcc
        f = (diffuse_cos + spec) * cc_att + cc_cos
        if p_diff > 0:
            pdf += p_diff * nl / math.pi
        if p_spec > 0:
            w = p_spec
            if p_trans > 0:
                ci = min(max(vh, 0.0), 1.0)
                if (etai / etat) * math.sqrt(max(0.0, 1 - ci * ci)) >= 1:
                    w += p_trans
            pdf += w * (_G1(nv, a2) * D * max(0.0, vh)) / max(4 * vh, 1e-7)
        if p_cc > 0:
            pdf += p_cc * (_G1(nv, cc_a2) * _D(nh, cc_a2) * max(0.0, vh)) / max(4 * vh, 1e-7)
    elif nl < 0 and (trans > 0 or p_trans > 0):
        Hv = -(etai * V + etat * L)
        H = Hv / np.linalg.norm(Hv)
        if float(H @ no) < 0:
            H = -H
        nh = max(float(no @ H), 0.0)
        vh, lh = float(V @ H), float(L @ H)
        if vh * lh < 0:
            D = _D(nh, a2)
            den = etai * vh + etat * lh
            if trans > 0:
                Fd = _fresnel_dielectric(vh, etai, etat)
                btdf = (abs(vh) * abs(lh) * etat * etat * (1 - Fd) * D * _G2u(nv, abs(nl), a2)
                        / max(den * den, 1e-7) * (1 + alpha * 0.25))
                cc_att = 1 - mat["clearcoat"] * Fcc if (mat["clearcoat"] > 0 and entering) else 1.0
                f = np.full(3, trans * (1 - metallic) * btdf * cc_att)
            if p_trans > 0:
                pdf += p_trans * (_G1(nv, a2) * D * max(0.0, vh)) * (etat * etat * abs(lh)) / max(den * den, 1e-7)
    return f, max(pdf, 1e-7)


# ------------------------------------------------------------------ OBJ (tracer.js:949-1021)
_FLOAT_RE = None


def _js_parse_float(s: str) -> float:
    import re
    global _FLOAT_RE
    if _FLOAT_RE is None:
        _FLOAT_RE = re.compile(r"[+-]?(Infinity|(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?)")
    m = _FLOAT_RE.match(s.lstrip(" \t\r\n\v\f"))
    if not m:
        return math.nan
    t = m.group(0)
    if t.lstrip("+-") == "Infinity":
        return -math.inf if t.startswith("-") else math.inf
    return float(t)


def _js_parse_int(s: str) -> float:
    s = s.lstrip(" \t\r\n\v\f")
    sign, i = 1.0, 0
    if s[:1] in ("+", "-"):
        sign = -1.0 if s[0] == "-" else 1.0
        i = 1
    base = 10
    if s[i:i + 2].lower() == "0x":
        base, i = 16, i + 2
    digits = "0123456789abcdef"[:base]
    v, n = 0, 0
    while i < len(s) and s[i].lower() in digits:
        v = v * base + digits.index(s[i].lower())
        i += 1
        n += 1
    return sign * v if n else math.nan


def _int32(x: float) -> float:
    if not math.isfinite(x):
        return 0.0
    m = math.fmod(math.trunc(x), 4294967296.0)
    if m < 0:
        m += 4294967296.0
    return m - 4294967296.0 if m >= 2147483648.0 else m


def _at(a, index: float) -> float:
    if not (index >= 0) or index != math.floor(index) or index >= len(a):
        return math.nan
    return float(np.float32(a[int(index)]))


def parse_obj(text: str) -> np.ndarray:
    """Model.parseOBJ + generateTriangles in plain Python with JavaScript semantics: n x 24
    float32 triangles (v0 v1 v2 n0 n1 n2 uv0 uv1 uv2)."""
    import re
    P, U, N, fp, fu, fn = [], [], [], [], [], []
    for line in text.split("\n"):
        parts = re.split(r"[ \t\r\n\v\f]+", line.strip(" \t\r\n\v\f"))
        part = lambda i: parts[i] if i < len(parts) else ""
        typ = parts[0]
        if typ == "v":
            P += [_js_parse_float(part(1)), _js_parse_float(part(2)), _js_parse_float(part(3))]
        elif typ == "vt":
            U += [_js_parse_float(part(1)), _js_parse_float(part(2))]
        elif typ == "vn":
            N += [_js_parse_float(part(1)), _js_parse_float(part(2)), _js_parse_float(part(3))]
        elif typ == "f":
            face = []
            for p in parts[1:]:
                idx = p.split("/")
                face.append((_js_parse_int(idx[0]) - 1,
                             _js_parse_int(idx[1]) - 1 if len(idx) > 1 and idx[1] else -1,
                             _js_parse_int(idx[2]) - 1 if len(idx) > 2 and idx[2] else -1))
            for i in range(1, len(face) - 1):
                for c in (face[0], face[i], face[i + 1]):
                    fp.append(c[0]); fu.append(c[1]); fn.append(c[2])
    out = np.zeros((len(fp) // 3, 24), np.float32)
    for t in range(len(fp) // 3):
        for c in range(3):
            ip, iu, iN = _int32(fp[t * 3 + c]), _int32(fu[t * 3 + c]), _int32(fn[t * 3 + c])
            for d in range(3):
                out[t, c * 3 + d] = _at(P, ip * 3 + d)
                out[t, 9 + c * 3 + d] = _at(N, iN * 3 + d)
            for d in range(2):
                out[t, 18 + c * 2 + d] = _at(U, iu * 2 + d)
    return out
