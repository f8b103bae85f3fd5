"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference checkout and numba installed,
naming the checkout with ``--reference DIR`` or the ``TOD_REFERENCE_DIR``
environment variable (default: /root/reference):

    python tests/golden/make_golden.py --reference /path/to/checkout

The reference's Numba kernels write their JIT cache next to their sources, so
the script copies the checkout to /tmp/refcopy and points NUMBA_CACHE_DIR at
/tmp/nbcache.  ``tod_core`` imports healpy at module level but its production
branch never calls it; a tiny stand-in module providing ``nside2npix`` lets it
import (healpy itself is not installed here).

Every fixture stores the exact inputs handed to the reference and the
reference's outputs; nothing at test time reads the reference checkout.
"""

from __future__ import annotations

import math
import os
import shutil
import sys
import types

REF = os.environ.get("TOD_REFERENCE_DIR", "/root/reference")
COPY = "/tmp/refcopy"
HERE = os.path.dirname(os.path.abspath(__file__))


def _import_reference():
    if not os.path.isdir(COPY):
        shutil.copytree(REF, COPY, ignore=shutil.ignore_patterns("__pycache__", "*.nbc", "*.nbi"))
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/nbcache")
    sys.path.insert(0, COPY)
    hp = types.ModuleType("healpy")
    hp.nside2npix = lambda nside: 12 * int(nside) ** 2
    sys.modules.setdefault("healpy", hp)


_import_reference()

import numba  # noqa: E402
import numpy as np  # noqa: E402

import numba_healpy as nh  # noqa: E402
import tod_bilinear as tb  # noqa: E402
import tod_nearest as tn  # noqa: E402
import tod_rotations as tr  # noqa: E402
import tod_core as tc  # noqa: E402
import tod_utils as tu  # noqa: E402
import beam_cluster as bc  # noqa: E402


def _unit(shape, rng):
    v = rng.standard_normal(shape)
    v /= np.linalg.norm(v, axis=-1, keepdims=True)
    return v.astype(np.float32)


def _random_params(B, rng, pole_safe=True):
    """Seeded random rotation parameters in the style of the reference tests
    (tests/test_tod_bilinear.py:62-94)."""
    ang1 = rng.uniform(0.0, math.pi, B).astype(np.float32)
    axes = _unit((B, 3), rng)
    if pole_safe:
        th = rng.uniform(0.1, math.pi - 0.1, B)
        ph = rng.uniform(0.0, 2 * math.pi, B)
        pts = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1)
        pts = pts.astype(np.float32)
    else:
        pts = _unit((B, 3), rng)
    ang2 = rng.uniform(0.0, 2 * math.pi, B).astype(np.float32)
    return (axes, np.cos(ang1).astype(np.float32), np.sin(ang1).astype(np.float32), pts,
            np.cos(ang2).astype(np.float32), np.sin(ang2).astype(np.float32))


def _pole_params(B, rng):
    """Boresights within a few pixels of the poles (identity recentre, random
    roll): exercises the north/south-cap stencil branches."""
    axes = np.tile(np.array([0.0, 0.0, 1.0], np.float32), (B, 1))
    cos_a = np.ones(B, np.float32)
    sin_a = np.zeros(B, np.float32)
    th = np.concatenate([rng.uniform(0.0, 0.05, B // 2), rng.uniform(math.pi - 0.05, math.pi, B - B // 2)])
    ph = rng.uniform(0, 2 * math.pi, B)
    pts = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1).astype(np.float32)
    ang2 = rng.uniform(0.0, 2 * math.pi, B).astype(np.float32)
    return axes, cos_a, sin_a, pts, np.cos(ang2).astype(np.float32), np.sin(ang2).astype(np.float32)


def _pole_beam(S, rng, radius):
    """Beam-frame vectors within `radius` of the +z pole (a realistic beam)."""
    r = radius * np.sqrt(rng.uniform(0, 1, S))
    a = rng.uniform(0, 2 * math.pi, S)
    return np.stack([np.sin(r) * np.cos(a), np.sin(r) * np.sin(a), np.cos(r)], -1).astype(np.float32)


@numba.njit(cache=False)
def _fused_stencils(vec_orig, axes, cos_a, sin_a, ax_pts, cos_p, sin_p, nside, pix, wgt):
    """Per-(b, s) stencil of the fused bilinear path, via the reference's own
    inlined helpers (tod_bilinear.py:312-352)."""
    B = axes.shape[0]
    S = vec_orig.shape[0]
    npix = 12 * nside * nside
    for b in range(B):
        for s in range(S):
            vx, vy, vz = tr._rodrigues_apply_one_jit(
                float(vec_orig[s, 0]), float(vec_orig[s, 1]), float(vec_orig[s, 2]),
                float(axes[b, 0]), float(axes[b, 1]), float(axes[b, 2]),
                float(cos_a[b]), float(sin_a[b]),
                float(ax_pts[b, 0]), float(ax_pts[b, 1]), float(ax_pts[b, 2]),
                float(cos_p[b]), float(sin_p[b]))
            z = max(-1.0, min(1.0, vz))
            phi_w = math.atan2(vy, vx)
            if phi_w < 0.0:
                phi_w += 2.0 * math.pi
            r = nh._ring_interp_with_angles_jit(nside, z, phi_w, npix)
            n = b * S + s
            pix[0, n] = r[0]
            pix[1, n] = r[1]
            pix[2, n] = r[2]
            pix[3, n] = r[3]
            wgt[0, n] = r[4]
            wgt[1, n] = r[5]
            wgt[2, n] = r[6]
            wgt[3, n] = r[7]


def kernel_cases():
    cases = {}
    specs = [
        # name, nside, B, S, C, comps, map dtype, pointing kind
        ("qu_n16", 16, 24, 40, 3, [0, 1, 2], np.float32, "random"),
        ("t_n16", 16, 24, 40, 1, [0], np.float32, "random"),
        ("iq_n8", 8, 20, 30, 2, [0, 1], np.float32, "random"),
        ("qu_n2", 2, 16, 25, 3, [0, 1, 2], np.float32, "random"),
        ("qu_n1", 1, 12, 10, 3, [0, 1, 2], np.float64, "random"),
        ("qu_n32_f64", 32, 20, 60, 3, [0, 1, 2], np.float64, "random"),
        ("qu_poles_n16", 16, 24, 40, 3, [0, 1, 2], np.float32, "poles"),
        ("qu_unsafe_n16", 16, 24, 40, 3, [0, 1, 2], np.float32, "unsafe"),
        ("qu_beam_n64", 64, 16, 200, 3, [0, 1, 2], np.float32, "beam"),
        ("uq_order_n16", 16, 16, 30, 3, [2, 0, 1], np.float32, "random"),
    ]
    for i, (name, nside, B, S, C, comps, mdt, kind) in enumerate(specs):
        rng = np.random.default_rng(1000 + i)
        if kind == "beam":
            vec = _pole_beam(S, rng, math.radians(2.0))
        else:
            vec = _unit((S, 3), rng)
        if kind == "poles":
            params = _pole_params(B, rng)
            vec = _pole_beam(S, rng, math.radians(8.0))
        elif kind == "unsafe":
            params = _random_params(B, rng, pole_safe=False)
        else:
            params = _random_params(B, rng)
        npix = 12 * nside * nside
        mp = rng.standard_normal((C, npix)).astype(mdt)
        bv = rng.uniform(0.1, 1.0, S).astype(np.float32)
        bv /= bv.sum()
        c_q = comps.index(1) if 1 in comps else -1
        c_u = comps.index(2) if 2 in comps else -1
        if c_q < 0 or c_u < 0:
            c_q_k, c_u_k = -1, -1
        else:
            c_q_k, c_u_k = c_q, c_u
        tod_bil = rng.standard_normal((C, B))  # non-zero start: the kernel accumulates (+=)
        tod_near = tod_bil.copy()
        tod0 = tod_bil.copy()
        tb._gather_accum_fused_jit(vec, *params, nside, mp, bv, B, S, tod_bil, c_q_k, c_u_k)
        tn._gather_accum_nearest_jit(vec, *params, nside, mp, bv, B, S, tod_near, c_q_k, c_u_k)
        pix = np.empty((4, B * S), np.int64)
        wgt = np.empty((4, B * S), np.float64)
        _fused_stencils(vec, *params, nside, pix, wgt)
        cases[name] = dict(
            nside=nside, B=B, S=S, c_q=c_q_k, c_u=c_u_k, vec_orig=vec, axes=params[0],
            cos_a=params[1], sin_a=params[2], ax_pts=params[3], cos_p=params[4],
            sin_p=params[5], mp_stacked=mp, beam_vals=bv, tod_init=tod0,
            tod_bilinear=tod_bil, tod_nearest=tod_near, stencil_pix=pix, stencil_wgt=wgt)
    return cases


def healpix_cases():
    rng = np.random.default_rng(7)
    out = {}
    for nside in (1, 2, 4, 16, 128, 1024):
        n = 1500
        theta = np.concatenate([rng.uniform(0, math.pi, n - 400), rng.uniform(0, 0.02, 100),
                                rng.uniform(math.pi - 0.02, math.pi, 100), np.zeros(1),
                                np.full(1, math.pi), rng.uniform(0.8, 0.85, 198)])
        phi = rng.uniform(0, 2 * math.pi, theta.shape[0])
        pix, wgt = nh.get_interp_weights_numba(nside, theta, phi)
        a2p = np.array([nh._ang2pix_ring_jit(nside, t, p) for t, p in zip(theta, phi)], np.int64)
        npix = 12 * nside * nside
        pp = np.unique(np.concatenate([np.arange(min(npix, 64)), rng.integers(0, npix, 600),
                                       np.arange(max(0, npix - 64), npix)]))
        th2, ph2 = nh.pix2ang_numba(nside, pp)
        out[f"n{nside}"] = dict(nside=nside, theta=theta, phi=phi, pix=pix, wgt=wgt, ang2pix=a2p,
                                pix2ang_pix=pp, pix2ang_theta=th2, pix2ang_phi=ph2)
    return out


def spin2_case():
    rng = np.random.default_rng(11)
    n = 3000
    z1 = rng.uniform(-1, 1, n)
    z2 = np.clip(z1 + rng.normal(0, 0.05, n), -1, 1)
    p1 = rng.uniform(0, 2 * math.pi, n)
    p2 = (p1 + rng.normal(0, 0.05, n)) % (2 * math.pi)
    z2[:50] = z1[:50]
    p2[:50] = p1[:50]
    s1 = np.sqrt(np.maximum(0, 1 - z1 * z1))
    s2 = np.sqrt(np.maximum(0, 1 - z2 * z2))
    c2 = np.empty(n)
    s2d = np.empty(n)
    for i in range(n):
        c2[i], s2d[i] = tb._spin2_cos2d_sin2d_jit(z1[i], s1[i], p1[i], z2[i], s2[i], p2[i])
    return dict(z_pix=z1, sth_pix=s1, phi_pix=p1, z_pts=z2, sth_pts=s2, phi_pts=p2, c2d=c2, s2d=s2d)


def rotation_case():
    """precompute_rotation_vector_batch + _rotation_params on a small pole-centred
    beam grid and a float32 spin scan (sample_based_tod_generation_gridint.py:277-281)."""
    rng = np.random.default_rng(21)
    H = W = 9
    ra = np.linspace(-0.01, 0.01, W)[None, :].repeat(H, 0)
    dec = (math.pi / 2 - np.linspace(0.0, 0.02, H))[:, None].repeat(W, 1)
    dec[H // 2, W // 2] = math.pi / 2
    ra[H // 2, W // 2] = 0.0
    n = 500
    t = np.arange(n) / 100.0
    theta = (math.pi / 2 + 0.87 * np.sin(2 * math.pi * t / 60.0)).astype(np.float32)
    phi = ((2 * math.pi * t / 86400.0) % (2 * math.pi)).astype(np.float32)
    phi[:20] = rng.uniform(0, 2 * math.pi, 20).astype(np.float32)
    theta[20:40] = rng.uniform(0, math.pi, 20).astype(np.float32)
    psi = (phi.astype(np.float64) + math.pi / 2).astype(np.float32)
    rot, beta = tr.precompute_rotation_vector_batch(ra, dec, phi, theta)
    psis = -beta + psi
    axes, cos_a, sin_a, pts, cos_p, sin_p = tr._rotation_params(rot, phi, theta, psis)
    return dict(ra=ra, dec=dec, phi=phi, theta=theta, psi=psi, rot_vecs=rot, beta=beta,
                psis=psis, axes=axes, cos_a=cos_a, sin_a=sin_a, ax_pts=pts, cos_p=cos_p,
                sin_p=sin_p)


def core_case():
    """tod_core.beam_tod_batch end to end (float32 dict) for both modes."""
    rng = np.random.default_rng(31)
    nside = 16
    npix = 12 * nside * nside
    rc = rotation_case()
    B = 64
    sel = slice(40, 40 + B)
    vec = _pole_beam(50, rng, math.radians(6.0))
    bv = rng.uniform(0.1, 1.0, 50).astype(np.float32)
    bv /= bv.sum()
    mp = rng.standard_normal((3, npix)).astype(np.float32)
    out = dict(nside=nside, rot_vecs=rc["rot_vecs"][sel], phi=rc["phi"][sel], theta=rc["theta"][sel],
               psis=rc["psis"][sel], vec_orig=vec, beam_vals=bv, maps=mp)
    for comps, tag in (([0, 1, 2], "iqu"), ([0, 1], "iq"), ([2], "u")):
        data = dict(vec_orig=vec, beam_vals=bv, comp_indices=comps,
                    mp_stacked=np.ascontiguousarray(mp[comps]))
        for mode in ("bilinear", "nearest"):
            res = tc.beam_tod_batch(nside, list(mp), data, rc["rot_vecs"][sel], rc["phi"][sel],
                                    rc["theta"][sel], rc["psis"][sel], interp_mode=mode)
            out[f"{tag}_{mode}"] = np.stack([res[c] for c in comps])
    return out


def beam_prep_case():
    """dB-threshold beam selection (tod_utils.py:254-297 +
    sample_based_tod_generation_gridint.py:131-136) and hybrid clustering split
    (beam_cluster.py:307-397)."""
    rng = np.random.default_rng(41)
    H = W = 41
    x = np.linspace(-1, 1, W)
    X, Y = np.meshgrid(x, x)
    beam = np.exp(-(X ** 2 + 1.3 * Y ** 2) / 0.08) + 1e-6 * rng.uniform(0, 1, (H, W))
    out = {"beam": beam}
    for cut in (0.9, 0.99, 0.999, 1.0):
        db = tu._compute_dB_threshold_from_power(beam, cut)
        sel = 10 * np.log10(np.abs(beam) + 1e-30) > db
        out[f"db_{cut}"] = np.float64(db)
        out[f"sel_{cut}"] = sel
    sel = out["sel_0.99"]
    ra = X * 0.02
    dec = math.pi / 2 - Y * 0.02
    th = math.pi / 2 - dec
    vec = np.stack([np.sin(th) * np.cos(ra), np.sin(th) * np.sin(ra), np.cos(th)], -1)[sel].astype(np.float32)
    bv = beam[sel].astype(np.float32)
    bv /= bv.sum()
    for tf, k in ((0.05, 20), (0.2, 10000), (0.5, 7)):
        vo, bo, lab = bc.cluster_beam_pixels(vec, bv, n_clusters=k, tail_fraction=tf, verbose=False)
        out[f"cl_{tf}_{k}_vec"] = vo
        out[f"cl_{tf}_{k}_bv"] = bo
        out[f"cl_{tf}_{k}_labels"] = lab
    out["cl_vec_in"] = vec
    out["cl_bv_in"] = bv
    return out


def clusters_case():
    """cluster_beam_pixels (beam_cluster.py:215-397) on larger inputs: full
    mode and hybrid mode on a pixelised Gaussian beam, full mode on a
    power-law annulus with an azimuthal modulation (a far-sidelobe tail)."""
    out = {}
    nside = 512
    # pixel centres of RING rings 1..n (north cap) as unit vectors
    th, ph = [], []
    for i in range(1, 60):
        z = 1.0 - i * i / (3.0 * nside * nside)
        j = np.arange(4 * i)
        th.append(np.full(4 * i, math.acos(z)))
        ph.append((j + 0.5) * (math.pi / (2 * i)))
    th = np.concatenate(th)
    ph = np.concatenate(ph)
    vec = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1)
    g = np.exp(-0.5 * (th / 0.02) ** 2) * (1 + 0.3 * np.cos(2 * ph))
    sel = g > 1e-3 * g.max()
    gv = vec[sel].astype(np.float32)
    gb = (g[sel] / g[sel].sum()).astype(np.float32)
    ring = (th > 0.05) & (th < 0.1)
    tv = vec[ring].astype(np.float32)
    tb = (th[ring] ** -3.0 * (1 + 0.08 * np.cos(3 * ph[ring] + 0.4)))
    tb = (tb / tb.sum()).astype(np.float32)
    cases = {"gauss_full_64": (gv, gb, 64, None), "gauss_hybrid_40": (gv, gb, 40, 0.3),
             "annulus_full_200": (tv, tb, 200, None), "gauss_full_3": (gv, gb, 3, None)}
    for name, (v, b, k, tf) in cases.items():
        vo, bo, lab = bc.cluster_beam_pixels(v, b, n_clusters=k, tail_fraction=tf, verbose=False)
        out[f"{name}__vec_in"] = v
        out[f"{name}__bv_in"] = b
        out[f"{name}__k"] = np.int64(k)
        out[f"{name}__tail_fraction"] = np.float64(-1.0 if tf is None else tf)
        out[f"{name}__vec"] = vo
        out[f"{name}__bv"] = bo
        out[f"{name}__labels"] = lab
    return out


def main():
    global REF
    if "--reference" in sys.argv:
        REF = sys.argv[sys.argv.index("--reference") + 1]
    if "--only-clusters" in sys.argv:
        np.savez_compressed(os.path.join(HERE, "clusters.npz"), **clusters_case())
        return
    np.savez_compressed(os.path.join(HERE, "kernels.npz"),
                        **{f"{c}__{k}": v for c, d in kernel_cases().items() for k, v in d.items()})
    np.savez_compressed(os.path.join(HERE, "healpix.npz"),
                        **{f"{c}__{k}": v for c, d in healpix_cases().items() for k, v in d.items()})
    np.savez_compressed(os.path.join(HERE, "spin2.npz"), **spin2_case())
    np.savez_compressed(os.path.join(HERE, "rotations.npz"), **rotation_case())
    np.savez_compressed(os.path.join(HERE, "core.npz"), **core_case())
    np.savez_compressed(os.path.join(HERE, "beam_prep.npz"), **beam_prep_case())
    np.savez_compressed(os.path.join(HERE, "clusters.npz"), **clusters_case())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
