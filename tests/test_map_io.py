"""CPU tests of the FITS readers and writers that replace healpy.read_map and
tod_io.load_beam (pixell): byte layout, round trips, NESTED -> RING
reordering checked against pixel geometry, the CAR beam coordinates and the
error paths."""

import numpy as np
import pytest

import oracle
from tod_generation_mapbased_beam_b200 import map_io as MI


def _angdist(t1, p1, t2, p2):
    c = np.sin(t1) * np.sin(t2) * np.cos(p1 - p2) + np.cos(t1) * np.cos(t2)
    return np.arccos(np.clip(c, -1.0, 1.0))


@pytest.mark.parametrize("nside", [1, 2, 4, 16, 64])
def test_nest2ring_is_a_permutation_with_inverse(nside):
    npix = 12 * nside * nside
    ip = np.arange(npix)
    r = MI.nest2ring(nside, ip)
    assert np.array_equal(np.sort(r), ip)
    assert np.array_equal(MI.ring2nest(nside, r), ip)
    if nside == 1:
        assert np.array_equal(r, ip)  # the 12 base pixels are numbered alike


@pytest.mark.parametrize("nside", [2, 8, 32, 128])
def test_nest2ring_matches_the_hierarchy_geometrically(nside):
    """The four NESTED children of a pixel lie inside it: each child's centre
    (RING index -> centre by the oracle's pix2ang) is within one parent pixel
    size of the parent's centre, and siblings sit around their mean."""
    oracle.build()
    npix = 12 * nside * nside
    ip = np.arange(npix)
    tc, pc = oracle.pix2ang(nside, MI.nest2ring(nside, ip))
    tp, pp = oracle.pix2ang(nside // 2, MI.nest2ring(nside // 2, ip // 4))
    size_parent = np.sqrt(4 * np.pi / (npix // 4))
    d = _angdist(tc, pc, tp, pp)
    assert d.max() < 0.8 * size_parent
    # a wrong in-face bit order would move children across the parent
    sib = _angdist(tc.reshape(-1, 4)[:, 0], pc.reshape(-1, 4)[:, 0], tc.reshape(-1, 4)[:, 3], pc.reshape(-1, 4)[:, 3])
    assert sib.max() < 1.2 * size_parent


def test_write_read_round_trip_and_byte_layout(tmp_path):
    nside = 16
    rng = np.random.default_rng(0)
    m = rng.standard_normal((3, 12 * nside * nside))
    p = str(tmp_path / "sky.fits")
    MI.write_map(p, m, dtype=np.float32)
    raw = open(p, "rb").read()
    assert len(raw) % 2880 == 0
    assert raw[:30] == b"SIMPLE  =                    T"
    ext = raw[2880:2880 * 2].decode("ascii")
    assert "XTENSION= 'BINTABLE'" in ext and "TFORM1  = '1024E   '" in ext
    assert "ORDERING= 'RING    '" in ext and "NSIDE   =                   16" in ext
    assert "TTYPE2  = 'Q_POLARISATION'" in ext
    got = MI.read_map(p, field=(0, 1, 2))
    assert got.shape == (3, 12 * nside * nside) and got.dtype == np.float32
    assert np.array_equal(got, m.astype(np.float32))
    one = MI.read_map(p)  # default field 0: one (npix,) map
    assert one.shape == (12 * nside * nside,) and np.array_equal(one, got[0])
    assert MI.read_map(p, field=2, dtype=np.float64).dtype == np.float64
    # the reference's use: float32 copies of the three fields
    mp = [x.astype(np.float32) for x in MI.read_map(p, field=(0, 1, 2))]
    assert len(mp) == 3 and all(np.array_equal(a, b) for a, b in zip(mp, got))


def test_nested_file_is_reordered_to_ring(tmp_path):
    nside = 8
    npix = 12 * nside * nside
    ring = np.arange(npix, dtype=np.float64)
    nested = ring[MI.nest2ring(nside, np.arange(npix))]  # NESTED pixel i holds RING value nest2ring(i)
    p = str(tmp_path / "nest.fits")
    MI.write_map(p, nested, nest=True)
    assert "ORDERING= 'NESTED  '" in open(p, "rb").read()[2880:5760].decode("ascii")
    assert np.array_equal(MI.read_map(p), ring)
    assert np.array_equal(MI.read_map(p, nest=True), nested)
    q = str(tmp_path / "ring.fits")
    MI.write_map(q, ring)
    assert np.array_equal(MI.read_map(q, nest=True), nested)


def test_small_maps_one_element_per_row(tmp_path):
    p = str(tmp_path / "n1.fits")
    MI.write_map(p, np.arange(12.0), dtype=np.float64)  # 12 pixels: not a multiple of 1024
    assert "TFORM1  = '1D      '" in open(p, "rb").read()[2880:5760].decode("ascii")
    assert np.array_equal(MI.read_map(p), np.arange(12.0))


def test_read_map_errors(tmp_path):
    p = str(tmp_path / "m.fits")
    MI.write_map(p, np.zeros((2, 48)))
    with pytest.raises(ValueError, match="no field"):
        MI.read_map(p, field=(0, 2))
    with pytest.raises(ValueError, match="no HDU"):
        MI.read_map(p, hdu=5)
    with pytest.raises(OSError):
        MI.write_map(p, np.zeros(48))
    with pytest.raises(ValueError, match="power of 2"):
        MI.nest2ring(3, [0])
    with pytest.raises(ValueError, match="12 nside"):
        MI.write_map(str(tmp_path / "bad.fits"), np.zeros(50))


def test_load_beam_car_coordinates(tmp_path):
    """Offsets from the grid-centre pixel, bound as the reference binds
    pixell's posmap() = [dec, ra]: first the declination offsets (varying
    along rows), then the right-ascension offsets (along columns)."""
    H, W = 9, 13
    dx, dy = -0.02, 0.03  # degrees
    rng = np.random.default_rng(1)
    beam = rng.uniform(0.0, 1.0, (1, H, W))
    MI.write_beam(str(tmp_path / "b.fits"), beam, (dx, dy), crval_deg=(10.0, 0.0))
    ra, dec, pix = MI.load_beam(str(tmp_path) + "/", "b.fits")
    assert ra.shape == dec.shape == pix.shape == (H, W)
    assert np.array_equal(pix, beam[0])
    yy, xx = np.mgrid[0:H, 0:W]
    np.testing.assert_allclose(ra, np.radians((yy - H // 2) * dy), rtol=0, atol=1e-15)
    np.testing.assert_allclose(dec, np.radians((xx - W // 2) * dx), rtol=0, atol=1e-15)
    assert ra[H // 2, W // 2] == 0.0 and dec[H // 2, W // 2] == 0.0


def test_load_beam_rejects_oblique_car(tmp_path):
    p = tmp_path / "b.fits"
    MI.write_beam(str(p), np.ones((1, 3, 3)), (0.1, 0.1))
    raw = bytearray(open(p, "rb").read())
    i = raw.find(b"CRVAL2  =")
    raw[i:i + 80] = MI._card("CRVAL2", 45.0).encode("ascii")
    open(p, "wb").write(bytes(raw))
    with pytest.raises(NotImplementedError):
        MI.load_beam(str(tmp_path) + "/", "b.fits")


def test_prepare_beam_data_and_load_sky(tmp_path):
    """The driver's beam preparation from FITS files (gridint.py:92-159) and
    the float32 sky load (gridint.py:406-408): entries per distinct file,
    shared components grouped, the strict dB selection, sum normalisation and
    float32 unit vectors -- the same values as the steps done by hand."""
    from tod_generation_mapbased_beam_b200 import driver
    from tod_generation_mapbased_beam_b200 import workloads as W

    H = W_ = 41
    yy, xx = np.mgrid[0:H, 0:W_]
    r2 = ((yy - H // 2) ** 2 + ((xx - W_ // 2) * 1.2) ** 2) * 0.02 ** 2
    bI = np.exp(-r2 / (2 * 0.1 ** 2))[None]
    bU = 0.01 * bI * np.sin(2 * np.arctan2(yy - H // 2, xx - W_ // 2))[None]
    folder = str(tmp_path) + "/"
    MI.write_beam(folder + "bI.fits", bI, (0.02, 0.02))
    MI.write_beam(folder + "bU.fits", bU, (0.02, 0.02))
    data = driver.prepare_beam_data(["bI.fits", "bI.fits", "bU.fits"], folder,
                                    {"bI.fits": 0.99, "bU.fits": 0.98})
    assert list(data) == ["bI.fits", "bU.fits"]
    assert data["bI.fits"]["comp_indices"] == [0, 1] and data["bU.fits"]["comp_indices"] == [2]
    for bf, cut in (("bI.fits", 0.99), ("bU.fits", 0.98)):
        ra, dec, pm = MI.load_beam(folder, bf)
        sel = W.select_beam_pixels(pm, cut)
        e = data[bf]
        assert np.array_equal(e["sel"], sel) and e["n_sel"] == int(sel.sum())
        bv = pm[sel].astype(np.float32)
        bv /= bv.sum()
        assert e["beam_vals"].dtype == np.float32 and np.array_equal(e["beam_vals"], bv)
        th = np.pi / 2 - dec
        v = np.stack([np.sin(th) * np.cos(ra), np.sin(th) * np.sin(ra), np.cos(th)], -1)[sel].astype(np.float32)
        assert np.array_equal(e["vec_orig"], v)
    nside = 8
    sky = np.random.default_rng(3).standard_normal((3, 12 * nside * nside))
    MI.write_map(folder + "sky.fits", sky)
    mp = driver.load_sky(folder + "sky.fits")
    assert len(mp) == 3 and all(m.dtype == np.float32 for m in mp)
    assert all(np.array_equal(m, s.astype(np.float32)) for m, s in zip(mp, sky))


def _image_file(path, data_be, bitpix, extra_cards=()):
    """A primary-HDU FITS image with the given big-endian data and cards."""
    cards = [MI._card("SIMPLE", True), MI._card("BITPIX", bitpix), MI._card("NAXIS", data_be.ndim)]
    for i, n in enumerate(reversed(data_be.shape)):
        cards.append(MI._card(f"NAXIS{i + 1}", int(n)))
    cards += [MI._card("CTYPE1", "RA---CAR"), MI._card("CTYPE2", "DEC--CAR"), MI._card("CDELT1", -0.05),
              MI._card("CDELT2", 0.05), MI._card("CRPIX1", 3.0), MI._card("CRPIX2", 2.0)]
    cards += list(extra_cards)
    raw = data_be.tobytes()
    with open(path, "wb") as f:
        f.write(MI._header_bytes(cards))
        f.write(raw)
        f.write(MI._pad(len(raw)))


def test_load_beam_scaled_integer_and_2d_images(tmp_path):
    """BSCALE / BZERO integer images are scaled like FITS readers do; a 2-D
    image gives map[0] = its first row, as the reference's map[0] does."""
    vals = np.arange(20, dtype=np.int16).reshape(1, 4, 5)
    _image_file(tmp_path / "i.fits", vals.astype(">i2"), 16, [MI._card("BSCALE", 0.5), MI._card("BZERO", 1.0)])
    ra, dec, pm = MI.load_beam(str(tmp_path) + "/", "i.fits")
    assert np.array_equal(pm, vals[0] * 0.5 + 1.0) and ra.shape == (4, 5)
    flat = np.linspace(0, 1, 12).reshape(3, 4)
    _image_file(tmp_path / "f.fits", flat.astype(">f4"), -32)
    ra, dec, pm = MI.load_beam(str(tmp_path) + "/", "f.fits")
    assert pm.shape == (4,) and np.array_equal(pm, flat[0].astype(np.float32))
    # offsets: declination along rows, right ascension along columns (pixell's posmap order)
    assert np.allclose(ra[:, 0], np.radians(0.05) * (np.arange(3) - 1))
    assert np.allclose(dec[0], np.radians(-0.05) * (np.arange(4) - 2))


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.int32, np.int64, np.int16])
def test_map_column_types(tmp_path, dtype):
    nside = 4
    m = (np.arange(12 * nside * nside) % 97 - 40).astype(dtype)
    p = str(tmp_path / "m.fits")
    MI.write_map(p, m, dtype=dtype)
    got = MI.read_map(p)
    assert got.dtype == np.dtype(dtype) and np.array_equal(got, m)
    assert MI.read_map(p, dtype=np.float64).dtype == np.float64
