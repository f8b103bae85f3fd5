"""FITS map input/output without healpy, astropy or pixell (none is installed
on the GPU hosts): drop-ins for the two readers the reference's driver calls
around the hot path.

* :func:`read_map` -- ``healpy.read_map(path, field=(0, 1, 2))`` as the driver
  loads the sky (sample_based_tod_generation_gridint.py:406-408): a HEALPix
  map stored as a FITS binary table (one column per Stokes component, any
  number of elements per row, big-endian float32/float64/integer columns),
  ``ORDERING`` RING or NESTED; NESTED maps are reordered to RING unless
  ``nest=True`` is asked for.
* :func:`load_beam` -- ``tod_io.load_beam`` (tod_io.py:6-36): a beam map as a
  FITS image in the plate-carree (CAR) projection, its pixel coordinates from
  the WCS keywords, offsets from the grid-centre pixel ``(H // 2, W // 2)``.
  Like the reference it unpacks ``ra, dec = posmap()`` where pixell's posmap is
  ``[dec, ra]``, so the first array returned holds the declination offsets and
  the second the right-ascension offsets; ``pixel_map`` is ``map[0]``.
* :func:`write_map` / :func:`write_beam` write the same formats (healpy's
  layout: 1024 elements per row, ``TTYPE`` TEMPERATURE / Q_POLARISATION /
  U_POLARISATION).

The FITS layout followed is the standard's (2880-byte blocks of 80-character
header cards, big-endian data); the NESTED -> RING map is the HEALPix
hierarchical-to-ring pixel index conversion (Gorski et al. 2005, ApJ 622, 759).
Only the plain CAR case (reference latitude CRVAL2 = 0, no rotation keywords)
is read: an oblique projection raises NotImplementedError.
"""

from __future__ import annotations

import os

import numpy as np

__all__ = ["read_map", "write_map", "load_beam", "write_beam", "nest2ring", "ring2nest", "UNSEEN"]

BLOCK = 2880
CARD = 80
UNSEEN = -1.6375e30

# TFORM letter -> big-endian numpy type
_TFORM = {"L": ">i1", "B": ">u1", "I": ">i2", "J": ">i4", "K": ">i8", "E": ">f4", "D": ">f8"}
_BITPIX = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}


# ---------------------------------------------------------------------------
# FITS headers and HDUs
# ---------------------------------------------------------------------------

def _value(text):
    t = text.strip()
    if t.startswith("'"):
        # string: up to the closing quote, '' is an escaped quote
        out, i = [], 1
        while i < len(t):
            if t[i] == "'":
                if i + 1 < len(t) and t[i + 1] == "'":
                    out.append("'")
                    i += 2
                    continue
                break
            out.append(t[i])
            i += 1
        return "".join(out).rstrip()
    v = t.split("/", 1)[0].strip()
    if v in ("T", "F"):
        return v == "T"
    if v == "":
        return None
    try:
        return int(v)
    except ValueError:
        return float(v.replace("D", "E").replace("d", "e"))


def _read_header(f):
    """Cards of one header as an ordered dict (keyword -> value)."""
    hdr = {}
    while True:
        block = f.read(BLOCK)
        if len(block) < BLOCK:
            raise ValueError("truncated FITS header")
        for k in range(0, BLOCK, CARD):
            card = block[k:k + CARD].decode("ascii", errors="replace")
            key = card[:8].strip()
            if key == "END":
                return hdr
            if card[8:10] == "= " and key:
                hdr[key] = _value(card[10:])


def _data_bytes(h):
    naxis = int(h.get("NAXIS", 0))
    if naxis == 0:
        return 0
    n = 1
    for i in range(1, naxis + 1):
        n *= int(h[f"NAXIS{i}"])
    n = abs(int(h["BITPIX"])) // 8 * int(h.get("GCOUNT", 1)) * (int(h.get("PCOUNT", 0)) + n)
    return (n + BLOCK - 1) // BLOCK * BLOCK


def _hdus(path):
    """[(header, data offset)] of every HDU of the file."""
    out = []
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        while f.tell() < size:
            h = _read_header(f)
            off = f.tell()
            out.append((h, off))
            f.seek(off + _data_bytes(h))
    return out


def _card(key, value=None, comment=""):
    if value is None:
        s = f"{key:<8}"
    else:
        if isinstance(value, bool):
            v = f"{'T' if value else 'F':>20}"
        elif isinstance(value, (int, np.integer)):
            v = f"{int(value):>20d}"
        elif isinstance(value, (float, np.floating)):
            v = f"{float(value):>20.16G}"
        else:
            v = "'" + str(value).replace("'", "''").ljust(8) + "'"
        s = f"{key:<8}= {v}" + (f" / {comment}" if comment else "")
    if len(s) > CARD:
        raise ValueError(f"FITS card too long: {s!r}")
    return s.ljust(CARD)


def _header_bytes(cards):
    text = "".join(cards) + "END".ljust(CARD)
    pad = (-len(text)) % BLOCK
    return (text + " " * pad).encode("ascii")


def _pad(nbytes):
    return b"\0" * ((-nbytes) % BLOCK)


# ---------------------------------------------------------------------------
# HEALPix NESTED <-> RING (Gorski et al. 2005)
# ---------------------------------------------------------------------------

_JRLL = np.array([2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4], dtype=np.int64)
_JPLL = np.array([1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7], dtype=np.int64)


def _compress_bits(v):
    """Every other bit of v (bits 0, 2, 4, ...) packed together."""
    v = v & 0x5555555555555555
    v = (v | (v >> 1)) & 0x3333333333333333
    v = (v | (v >> 2)) & 0x0F0F0F0F0F0F0F0F
    v = (v | (v >> 4)) & 0x00FF00FF00FF00FF
    v = (v | (v >> 8)) & 0x0000FFFF0000FFFF
    v = (v | (v >> 16)) & 0x00000000FFFFFFFF
    return v


def nest2ring(nside, ipnest):
    """RING index of NESTED pixels: base face and in-face (x, y) from the bit
    interleaving, ring number jr = jrll(face) nside - x - y - 1, in-ring index
    from jpll(face), the ring length and its half-pixel shift."""
    nside = int(nside)
    if nside < 1 or nside & (nside - 1):
        raise ValueError("NESTED ordering needs nside a power of 2")
    ip = np.asarray(ipnest, dtype=np.int64)
    npface = nside * nside
    face = ip // npface
    ipf = ip % npface
    ix = _compress_bits(ipf)
    iy = _compress_bits(ipf >> 1)
    jrt = ix + iy
    jpt = ix - iy
    jr = _JRLL[face] * nside - jrt - 1
    nl4 = 4 * nside
    ncap = 2 * nside * (nside - 1)
    npix = 12 * npface
    north = jr < nside
    south = jr > 3 * nside
    nr = np.where(north, jr, np.where(south, nl4 - jr, nside))
    n_before = np.where(north, 2 * nr * (nr - 1),
                        np.where(south, npix - 2 * (nr + 1) * nr, ncap + (jr - nside) * nl4))
    kshift = np.where(north | south, 0, (jr - nside) & 1)
    jp = (_JPLL[face] * nr + jpt + 1 + kshift) // 2
    jp = np.where(jp > nl4, jp - nl4, jp)
    jp = np.where(jp < 1, jp + nl4, jp)
    return n_before + jp - 1


def ring2nest(nside, ipring):
    """NESTED index of RING pixels (the inverse permutation of nest2ring)."""
    npix = 12 * int(nside) ** 2
    inv = np.empty(npix, dtype=np.int64)
    inv[nest2ring(nside, np.arange(npix, dtype=np.int64))] = np.arange(npix, dtype=np.int64)
    return inv[np.asarray(ipring, dtype=np.int64)]


# ---------------------------------------------------------------------------
# HEALPix maps
# ---------------------------------------------------------------------------

def read_map(filename, field=0, dtype=None, nest=False, hdu=1):
    """HEALPix map(s) of a FITS binary table, like ``healpy.read_map``.

    ``field``: column index or sequence of indices (0-based).  Returns one
    (npix,) array for an int ``field``, else an (nfield, npix) array.
    ``dtype``: the returned type (None: the column's own type, native byte
    order).  ``nest``: return NESTED ordering (default RING; the file's
    ``ORDERING`` keyword says what it holds).  ``hdu``: the extension number."""
    hdus = _hdus(filename)
    if hdu >= len(hdus):
        raise ValueError(f"{filename}: no HDU {hdu}")
    h, off = hdus[hdu]
    if h.get("XTENSION") != "BINTABLE":
        raise ValueError(f"{filename}: HDU {hdu} is not a binary table")
    nfields = int(h["TFIELDS"])
    cols = []
    for i in range(1, nfields + 1):
        form = str(h[f"TFORM{i}"]).strip()
        rep = int(form[:-1]) if len(form) > 1 else 1
        code = form[-1]
        if code not in _TFORM:
            raise ValueError(f"{filename}: unsupported column format {form!r}")
        cols.append((f"c{i}", _TFORM[code], (rep,)))
    rowdt = np.dtype(cols)
    if rowdt.itemsize != int(h["NAXIS1"]):
        raise ValueError(f"{filename}: row width {h['NAXIS1']} does not match the column formats")
    nrows = int(h["NAXIS2"])
    with open(filename, "rb") as f:
        f.seek(off)
        rows = np.frombuffer(f.read(rowdt.itemsize * nrows), dtype=rowdt, count=nrows)
    single = isinstance(field, (int, np.integer))
    fields = [int(field)] if single else [int(x) for x in field]
    ordering = str(h.get("ORDERING", "RING")).strip().upper()
    if ordering not in ("RING", "NESTED"):
        raise ValueError(f"{filename}: unknown ORDERING {ordering!r}")
    maps = []
    for fi in fields:
        if not 0 <= fi < nfields:
            raise ValueError(f"{filename}: no field {fi} (the table has {nfields})")
        m = rows[f"c{fi + 1}"].reshape(-1)
        m = m.astype(m.dtype.newbyteorder("=") if dtype is None else dtype)
        maps.append(m)
    npix = maps[0].shape[0]
    nside = int(h.get("NSIDE", round(np.sqrt(npix / 12))))
    if 12 * nside * nside != npix:
        raise ValueError(f"{filename}: {npix} pixels is not 12 nside^2 for NSIDE {nside}")
    if ordering == "NESTED" and not nest:
        n2r = nest2ring(nside, np.arange(npix, dtype=np.int64))
        out = []
        for m in maps:
            r = np.empty_like(m)
            r[n2r] = m
            out.append(r)
        maps = out
    elif ordering == "RING" and nest:
        n2r = nest2ring(nside, np.arange(npix, dtype=np.int64))
        maps = [m[n2r] for m in maps]
    return maps[0] if single else np.stack(maps)


_STD_NAMES = {1: ["TEMPERATURE"], 3: ["TEMPERATURE", "Q_POLARISATION", "U_POLARISATION"]}


def write_map(filename, m, nest=False, dtype=np.float64, column_names=None, overwrite=False,
              row_length=1024):
    """Write a HEALPix map (npix,) or maps (nmap, npix) in RING (or NESTED,
    ``nest=True``) ordering as healpy does: a primary header, one binary-table
    extension with ``row_length`` elements of every map per row."""
    if os.path.exists(filename) and not overwrite:
        raise OSError(f"{filename} exists (overwrite=False)")
    maps = np.atleast_2d(np.asarray(m))
    nmap, npix = maps.shape
    nside = int(round(np.sqrt(npix / 12)))
    if 12 * nside * nside != npix:
        raise ValueError(f"{npix} pixels is not 12 nside^2")
    dt = np.dtype(dtype)
    code = {np.dtype(np.float32): "E", np.dtype(np.float64): "D", np.dtype(np.int32): "J",
            np.dtype(np.int64): "K", np.dtype(np.int16): "I"}[dt]
    rep = row_length if npix % row_length == 0 else 1
    nrows = npix // rep
    names = column_names or _STD_NAMES.get(nmap, [f"COLUMN{i + 1}" for i in range(nmap)])
    rowdt = np.dtype([(f"c{i}", dt.newbyteorder(">"), (rep,)) for i in range(nmap)])
    rows = np.empty(nrows, dtype=rowdt)
    for i in range(nmap):
        rows[f"c{i}"] = maps[i].astype(dt).reshape(nrows, rep)
    prim = [_card("SIMPLE", True), _card("BITPIX", 8), _card("NAXIS", 0), _card("EXTEND", True)]
    ext = [_card("XTENSION", "BINTABLE"), _card("BITPIX", 8), _card("NAXIS", 2),
           _card("NAXIS1", rowdt.itemsize), _card("NAXIS2", nrows), _card("PCOUNT", 0), _card("GCOUNT", 1),
           _card("TFIELDS", nmap)]
    for i in range(nmap):
        ext += [_card(f"TTYPE{i + 1}", names[i]), _card(f"TFORM{i + 1}", f"{rep}{code}")]
    ext += [_card("PIXTYPE", "HEALPIX"), _card("ORDERING", "NESTED" if nest else "RING"),
            _card("NSIDE", nside), _card("FIRSTPIX", 0), _card("LASTPIX", npix - 1),
            _card("INDXSCHM", "IMPLICIT"), _card("OBJECT", "FULLSKY")]
    data = rows.tobytes()
    with open(filename, "wb") as f:
        f.write(_header_bytes(prim))
        f.write(_header_bytes(ext))
        f.write(data)
        f.write(_pad(len(data)))


# ---------------------------------------------------------------------------
# CAR beam maps
# ---------------------------------------------------------------------------

def _image_hdu(path):
    """The first HDU holding an image of two or more axes (primary or IMAGE
    extension)."""
    for h, off in _hdus(path):
        is_image = "SIMPLE" in h or str(h.get("XTENSION", "")).strip() == "IMAGE"
        if is_image and int(h.get("NAXIS", 0)) >= 2:
            return h, off
    raise ValueError(f"{path}: no image HDU")


def _read_image(path):
    h, off = _image_hdu(path)
    naxis = int(h["NAXIS"])
    shape = tuple(int(h[f"NAXIS{i}"]) for i in range(naxis, 0, -1))  # C order: slowest axis first
    dt = np.dtype(_BITPIX[int(h["BITPIX"])])
    with open(path, "rb") as f:
        f.seek(off)
        a = np.frombuffer(f.read(dt.itemsize * int(np.prod(shape))), dtype=dt).reshape(shape)
    a = a.astype(dt.newbyteorder("="))
    bscale, bzero = h.get("BSCALE", 1.0), h.get("BZERO", 0.0)
    if bscale != 1.0 or bzero != 0.0:
        a = a * bscale + bzero
    return h, a


def car_posmap(h, shape):
    """[dec, ra] (radians) of every pixel (y, x) of a plain CAR image: the
    linear world coordinates CRVAL + (pixel + 1 - CRPIX) CDELT of the two
    celestial axes (degrees), pixell's order."""
    ct1, ct2 = str(h.get("CTYPE1", "")), str(h.get("CTYPE2", ""))
    if not (ct1.endswith("CAR") and ct2.endswith("CAR")):
        raise NotImplementedError(f"only the CAR projection is read (CTYPE {ct1!r}, {ct2!r})")
    if float(h.get("CRVAL2", 0.0)) != 0.0 or any(k in h for k in ("PC1_2", "PC2_1", "CD1_2", "CD2_1", "CROTA2")):
        raise NotImplementedError("oblique or rotated CAR headers are not supported")
    H, W = shape[-2], shape[-1]
    cdelt1 = float(h.get("CDELT1", h.get("CD1_1", 1.0)))
    cdelt2 = float(h.get("CDELT2", h.get("CD2_2", 1.0)))
    x = (np.arange(W, dtype=np.float64) + 1.0 - float(h.get("CRPIX1", 1.0))) * cdelt1 + float(h.get("CRVAL1", 0.0))
    y = (np.arange(H, dtype=np.float64) + 1.0 - float(h.get("CRPIX2", 1.0))) * cdelt2 + float(h.get("CRVAL2", 0.0))
    ra = np.broadcast_to(np.radians(x)[None, :], (H, W))
    dec = np.broadcast_to(np.radians(y)[:, None], (H, W))
    return np.stack([dec, ra])


def load_beam(folder_beam, filename):
    """Drop-in for ``tod_io.load_beam`` (tod_io.py:6-36): ``(ra, dec,
    pixel_map)`` of a CAR beam image, offsets from the grid-centre pixel
    ``(H // 2, W // 2)``.  ``ra, dec`` are bound as the reference binds
    pixell's ``posmap()`` (which is ``[dec, ra]``): ``ra`` holds the
    declination offsets and ``dec`` the right-ascension offsets.
    ``pixel_map`` is ``map[0]`` -- the first component of a (ncomp, H, W)
    beam (the first row of a 2-D image, as in the reference)."""
    h, a = _read_image(folder_beam + filename)
    pos = car_posmap(h, a.shape)
    ra, dec = np.array(pos[0]), np.array(pos[1])
    center_idx = (ra.shape[0] // 2, ra.shape[1] // 2)
    ra = ra - ra[center_idx]
    dec = dec - dec[center_idx]
    return ra, dec, np.array(a[0])


def write_beam(filename, beam, cdelt_deg, crval_deg=(0.0, 0.0), overwrite=False):
    """Write a beam map (ncomp, H, W) or (H, W) as a float64 CAR FITS image with
    pixel spacing ``cdelt_deg`` (dx, dy) and the grid-centre pixel (H // 2,
    W // 2) at ``crval_deg`` (ra, 0); CRVAL2 must be 0 (plain CAR)."""
    if os.path.exists(filename) and not overwrite:
        raise OSError(f"{filename} exists (overwrite=False)")
    a = np.asarray(beam, dtype=np.float64)
    H, W = a.shape[-2], a.shape[-1]
    if crval_deg[1] != 0.0:
        raise ValueError("plain CAR needs CRVAL2 = 0")
    cards = [_card("SIMPLE", True), _card("BITPIX", -64), _card("NAXIS", a.ndim)]
    for i, n in enumerate(reversed(a.shape)):
        cards.append(_card(f"NAXIS{i + 1}", int(n)))
    cards += [_card("CTYPE1", "RA---CAR"), _card("CTYPE2", "DEC--CAR"),
              _card("CRPIX1", float(W // 2 + 1)), _card("CRPIX2", float(H // 2 + 1)),
              _card("CRVAL1", float(crval_deg[0])), _card("CRVAL2", float(crval_deg[1])),
              _card("CDELT1", float(cdelt_deg[0])), _card("CDELT2", float(cdelt_deg[1])),
              _card("CUNIT1", "deg"), _card("CUNIT2", "deg")]
    data = a.astype(">f8").tobytes()
    with open(filename, "wb") as f:
        f.write(_header_bytes(cards))
        f.write(data)
        f.write(_pad(len(data)))
