"""Input formats of the search: NPZ archives of NPY arrays and SPOC FITS
light-curve products (src/io/npz.rs, src/io/fits.rs), and the assembly of
several input files into one set of observations with sector groups
(read_inputs, src/main.rs:50-132). Host code only: the values are decoded
to f64 as the reference does.
"""
from __future__ import annotations

import dataclasses
import math
import struct
import zipfile
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

# -- NPZ (src/io/npz.rs) ---------------------------------------------------------


@dataclasses.dataclass
class Array:
    shape: Tuple[int, ...]
    data: np.ndarray  # f64, flattened

    def __len__(self) -> int:
        return int(self.data.shape[0])


_NPY_KINDS = {"f8": "f8", "f4": "f4", "i8": "i8", "i4": "i4", "i2": "i2", "u1": "u1", "b1": "u1"}


def _usize(text: str) -> int:
    """A non-negative integer as the reference's usize parse reads it: an
    optional '+' and ASCII digits, below 2^64; its error texts otherwise."""
    digits = text[1:] if text.startswith("+") else text
    if not digits:
        raise ValueError("cannot parse integer from empty string")
    if not (digits.isascii() and digits.isdigit()):
        raise ValueError("invalid digit found in string")
    value = int(digits)
    if value >= 1 << 64:
        raise ValueError("number too large to fit in target type")
    return value


def _i64(text: str) -> Optional[int]:
    """A signed integer as the reference's i64 parse reads it (None where it fails)."""
    sign, digits = (-1, text[1:]) if text.startswith("-") else (1, text[1:] if text.startswith("+") else text)
    if not digits or not (digits.isascii() and digits.isdigit()):
        return None
    value = sign * int(digits)
    return value if -(1 << 63) <= value < (1 << 63) else None


def _header_value(header: str, key: str) -> Optional[str]:
    """The text after `key` up to the next comma (npz.rs:92-96)."""
    parts = header.split(key, 1)
    if len(parts) < 2:
        return None
    rest = parts[1].lstrip()
    end = rest.find(",")
    return None if end < 0 else rest[:end].strip()


def parse_npy(data: bytes) -> Array:
    """One NPY member decoded to f64 (npz.rs:17-90): dtypes f8, f4, i8, i4,
    i2, u1 and b1 in either byte order; C order only."""
    if len(data) < 10 or data[:6] != b"\x93NUMPY":
        raise ValueError("not an NPY file")
    if data[6] != 1 and len(data) < 12:
        raise ValueError("truncated NPY header")
    if data[6] == 1:
        header_len, offset = struct.unpack("<H", data[8:10])[0], 10
    else:
        header_len, offset = struct.unpack("<I", data[8:12])[0], 12
    header = data[offset:offset + header_len].decode("ascii")
    descr = _header_value(header, "'descr':")
    if descr is None:
        raise ValueError("NPY header without descr")
    fortran = _header_value(header, "'fortran_order':")
    if fortran is not None and fortran.startswith("True"):
        raise ValueError("fortran_order arrays are not supported")
    parts = header.split("'shape':", 1)
    if len(parts) < 2 or "(" not in parts[1] or ")" not in parts[1]:
        raise ValueError("NPY header without shape")
    inner = parts[1].split("(", 1)[1].split(")", 1)[0]
    shape = tuple(_usize(s) for s in (x.strip() for x in inner.split(",")) if s)
    count = math.prod(shape)  # exact; 1 for a scalar
    descr = descr.strip("'\"")
    little = not descr.startswith(">")
    kind = descr[1:]
    if kind not in _NPY_KINDS:
        raise ValueError(f"unsupported NPY dtype: {kind}")
    code = _NPY_KINDS[kind]
    dt = np.dtype(code).newbyteorder("<" if little else ">")
    body = data[offset + header_len:]
    if len(body) < count * dt.itemsize:
        raise ValueError("truncated NPY body")
    values = np.frombuffer(body, dtype=dt, count=count).astype(np.float64)
    return Array(shape, values)


def read_npz(path: str) -> Dict[str, Array]:
    """Every member of an NPZ archive, by name without '.npy' (npz.rs:98-113)."""
    out = {}
    with zipfile.ZipFile(path) as z:
        for name in z.namelist():
            key = name[:-4] if name.endswith(".npy") else name
            try:
                out[key] = parse_npy(z.read(name))
            except ValueError as e:
                raise ValueError(f"{path}:{key}: {e}") from None
    return out


# -- FITS (src/io/fits.rs) -----------------------------------------------------

BLOCK = 2880
DEFAULT_QUALITY_BITMASK = 17087  # fits.rs:214-217


@dataclasses.dataclass
class Header:
    cards: List[Tuple[str, str]]

    def get(self, key: str) -> Optional[str]:
        for k, v in self.cards:
            if k == key:
                return v
        return None

    def f64(self, key: str) -> Optional[float]:
        v = self.get(key)
        if v is None or "_" in v:  # the reference's f64 parse takes no digit separators
            return None
        try:
            return float(v.strip())
        except ValueError:
            return None

    def i64(self, key: str) -> Optional[int]:
        v = self.get(key)
        return None if v is None else _i64(v.strip())

    def text(self, key: str) -> Optional[str]:
        v = self.get(key)
        return None if v is None else v.strip().strip("'").strip()


@dataclasses.dataclass
class Column:
    name: str
    code: str
    repeat: int
    offset: int
    width: int


_WIDTH = {"D": 8, "K": 8, "E": 4, "J": 4, "I": 2, "B": 1, "L": 1, "A": 1}
_BE = {"D": ">f8", "E": ">f4", "J": ">i4", "K": ">i8", "I": ">i2"}


@dataclasses.dataclass
class Hdu:
    name: str
    header: Header
    data: bytes
    columns: List[Column]
    rows: int
    row_bytes: int
    naxes: List[int]

    def column(self, name: str) -> Optional[Column]:
        for c in self.columns:
            if c.name == name:
                return c
        return None

    def _cells(self, col: Column) -> np.ndarray:
        raw = np.frombuffer(self.data, dtype=np.uint8, count=self.rows * self.row_bytes).reshape(self.rows,
                                                                                                 self.row_bytes)
        cells = raw[:, col.offset:col.offset + col.repeat * col.width]
        if col.code in _BE:
            return np.ascontiguousarray(cells).view(_BE[col.code]).astype(np.float64).reshape(self.rows, col.repeat)
        return cells.astype(np.float64).reshape(self.rows, col.repeat)

    def column_f64(self, name: str) -> np.ndarray:
        """A scalar column (the first cell of each row) as f64 (fits.rs:194-198)."""
        col = self.column(name)
        if col is None:
            raise ValueError(f"missing column {name}")
        return self._cells(col)[:, 0].copy()

    def column_array(self, name: str) -> Tuple[np.ndarray, int]:
        """An array column, `repeat` values per row, row-major (fits.rs:200-211)."""
        col = self.column(name)
        if col is None:
            raise ValueError(f"missing column {name}")
        return self._cells(col).reshape(-1).copy(), col.repeat


def _parse_header(data: bytes, at: int) -> Tuple[Header, int]:
    """80-character cards up to END (fits.rs:53-97)."""
    cards = []
    pos = at
    while True:
        if pos + 80 > len(data):
            raise ValueError("truncated FITS header")
        card = data[pos:pos + 80].decode("ascii")
        pos += 80
        key = card[:8].strip()
        if key == "END":
            break
        if not key or key in ("COMMENT", "HISTORY"):
            continue
        value = ""
        if card[8:10] == "= ":
            rest = card[10:]
            if rest.lstrip().startswith("'"):
                start = rest.find("'")
                end = start + 1
                while end < len(rest):
                    if rest[end] == "'":
                        if end + 1 < len(rest) and rest[end + 1] == "'":
                            end += 2
                            continue
                        break
                    end += 1
                value = rest[start:min(end, len(rest) - 1) + 1]
            else:
                value = rest.split("/")[0].strip()
        cards.append((key, value))
    end = -(-(pos - at) // BLOCK) * BLOCK + at
    return Header(cards), end


def read_fits(path: str) -> List[Hdu]:
    """Every header-data unit of a FITS file (fits.rs:109-174)."""
    with open(path, "rb") as fh:
        data = fh.read()
    hdus: List[Hdu] = []
    pos = 0
    while pos + BLOCK <= len(data):
        header, start = _parse_header(data, pos)
        bitpix = header.i64("BITPIX")
        bitpix = 8 if bitpix is None else bitpix
        naxis = header.i64("NAXIS") or 0
        if not 0 <= naxis <= 999:
            raise ValueError(f"{path}: invalid NAXIS {naxis}")
        naxes = [header.i64(f"NAXIS{i}") or 0 for i in range(1, naxis + 1)]
        pcount = header.i64("PCOUNT") or 0
        name = header.text("EXTNAME")
        if name is None:
            name = "PRIMARY" if not hdus else ""
        if any(n < 0 for n in naxes) or pcount < 0:
            # the reference reads these as usize: a negative value wraps to a
            # unit larger than any file
            raise ValueError(f"{path}: truncated data unit {name}")
        size = 0 if naxis == 0 else math.prod(naxes) * (abs(bitpix) // 8)
        size += pcount
        columns, rows, row_bytes = [], 0, 0
        if header.text("XTENSION") == "BINTABLE":
            row_bytes = naxes[0] if naxes else 0
            rows = naxes[1] if len(naxes) > 1 else 0
            offset = 0
            for i in range(1, (header.i64("TFIELDS") or 0) + 1):
                form = header.text(f"TFORM{i}")
                if form is None:
                    raise ValueError(f"missing TFORM{i}")
                if not form:
                    raise ValueError("empty TFORM")
                code = form[-1]
                try:
                    repeat = _usize(form[:-1])
                except ValueError:
                    repeat = 1  # parse().unwrap_or(1), fits.rs
                if code not in _WIDTH:
                    raise ValueError(f"unsupported FITS column type {code}")
                columns.append(Column(header.text(f"TTYPE{i}") or "", code, repeat, offset, _WIDTH[code]))
                offset += repeat * _WIDTH[code]
        end = start + size
        if end > len(data):
            raise ValueError(f"{path}: truncated data unit {name}")
        hdus.append(Hdu(name, header, data[start:end], columns, rows, row_bytes, naxes))
        pos = start + -(-size // BLOCK) * BLOCK
    return hdus


def tan_world_to_pixel(h: Header, ra: float, dec: float) -> Optional[Tuple[float, float]]:
    """Zero-based pixel of (ra, dec) under a TAN projection (fits.rs:218-258)."""
    vals = [h.f64(k) for k in ("CRPIX1", "CRPIX2", "CRVAL1", "CRVAL2")]
    if any(v is None for v in vals):
        return None
    crpix1, crpix2, crval1, crval2 = vals
    cdelt1 = h.f64("CDELT1")
    cdelt2 = h.f64("CDELT2")
    cdelt1 = 1.0 if cdelt1 is None else cdelt1
    cdelt2 = 1.0 if cdelt2 is None else cdelt2
    cd = [h.f64(k) for k in ("CD1_1", "CD1_2", "CD2_1", "CD2_2")]
    if all(v is not None for v in cd):
        pc11, pc12, pc21, pc22 = cd
    else:
        def g(k, d):
            v = h.f64(k)
            return d if v is None else v
        pc11, pc12 = g("PC1_1", 1.0) * cdelt1, g("PC1_2", 0.0) * cdelt1
        pc21, pc22 = g("PC2_1", 0.0) * cdelt2, g("PC2_2", 1.0) * cdelt2
    d2r = math.pi / 180.0
    a0, d0 = crval1 * d2r, crval2 * d2r
    a, d = ra * d2r, dec * d2r
    cos_c = math.sin(d0) * math.sin(d) + math.cos(d0) * math.cos(d) * math.cos(a - a0)
    if cos_c <= 0.0:
        return None
    x = math.cos(d) * math.sin(a - a0) / cos_c / d2r
    y = (math.cos(d0) * math.sin(d) - math.sin(d0) * math.cos(d) * math.cos(a - a0)) / cos_c / d2r
    det = pc11 * pc22 - pc12 * pc21
    if det == 0.0:
        return None
    p1 = (pc22 * x - pc12 * y) / det
    p2 = (-pc21 * x + pc11 * y) / det
    return p1 + crpix1 - 1.0, p2 + crpix2 - 1.0


@dataclasses.dataclass
class StarParameters:
    radius: Optional[float] = None
    teff: Optional[float] = None
    logg: Optional[float] = None
    tmag: Optional[float] = None


@dataclasses.dataclass
class LightCurve:
    """One SPOC light-curve product after the default quality mask (fits.rs:260-275)."""
    tic: int
    sector: int
    time_bjd: np.ndarray
    flux: np.ndarray
    flux_err: np.ndarray
    centr1: np.ndarray
    centr2: np.ndarray
    crowdsap: Optional[float]
    star: StarParameters
    target_pixel: Optional[Tuple[float, float]]
    points_total: int


def read_light_curve(path: str) -> LightCurve:
    """read_light_curve (fits.rs:284-333): PDCSAP flux of the LIGHTCURVE
    extension, rows with a clear default quality mask and finite time and
    flux, times in BJD."""
    hdus = read_fits(path)
    if not hdus:
        raise ValueError("empty FITS")
    primary = hdus[0]
    table = next((h for h in hdus if h.name == "LIGHTCURVE"), None)
    if table is None:
        raise ValueError("no LIGHTCURVE extension")
    aperture = next((h for h in hdus if h.name == "APERTURE"), None)
    bjd_ref = (table.header.f64("BJDREFI") or 0.0) + (table.header.f64("BJDREFF") or 0.0)
    time = table.column_f64("TIME")
    flux = table.column_f64("PDCSAP_FLUX")
    flux_err = table.column_f64("PDCSAP_FLUX_ERR")
    c1 = table.column_f64("MOM_CENTR1")
    c2 = table.column_f64("MOM_CENTR2")
    quality = table.column_f64("QUALITY")
    keep = ((quality.astype(np.int64) & DEFAULT_QUALITY_BITMASK) == 0) & np.isfinite(time) & np.isfinite(flux)
    target = None
    if aperture is not None:
        ra, dec = primary.header.f64("RA_OBJ"), primary.header.f64("DEC_OBJ")
        if ra is not None and dec is not None:
            xy = tan_world_to_pixel(aperture.header, ra, dec)
            c1p, c2p = aperture.header.f64("CRVAL1P"), aperture.header.f64("CRVAL2P")
            if xy is not None and c1p is not None and c2p is not None:
                target = (xy[0] + c1p, xy[1] + c2p)
    return LightCurve(
        tic=primary.header.i64("TICID") or 0, sector=primary.header.i64("SECTOR") or 0,
        time_bjd=time[keep] + bjd_ref, flux=flux[keep], flux_err=flux_err[keep], centr1=c1[keep], centr2=c2[keep],
        crowdsap=table.header.f64("CROWDSAP"),
        star=StarParameters(primary.header.f64("RADIUS"), primary.header.f64("TEFF"), primary.header.f64("LOGG"),
                            primary.header.f64("TESSMAG")),
        target_pixel=target, points_total=table.rows)


# -- several files to one set of observations (src/main.rs:50-132) ---------------


@dataclasses.dataclass
class Observations:
    time: np.ndarray
    flux: np.ndarray
    err: Optional[np.ndarray]
    group: np.ndarray  # one label per (file, sector)


def read_inputs(paths: Sequence[str]) -> Observations:
    """Concatenates the inputs; every (file, sector) pair gets its own group.
    FITS products give flux_err; NPZ files need time_bjd and flux and may give
    flux_err (all files or none) and a scalar or per-point sector."""
    time, flux, group = [], [], []
    err: Optional[List[np.ndarray]] = None
    groups: Dict[Tuple[int, int], int] = {}

    def label(index: int, sector: int) -> int:
        return groups.setdefault((index, sector), len(groups))

    for index, path in enumerate(paths):
        if path.endswith(".fits") or path.endswith(".fits.gz"):
            lc = read_light_curve(path)
            if index == 0:
                err = []
            if err is None:
                raise ValueError("all input files must either provide flux_err or omit it")
            err.append(lc.flux_err)
            time.append(lc.time_bjd)
            flux.append(lc.flux)
            group.append(np.full(lc.time_bjd.shape[0], label(index, lc.sector), dtype=np.int64))
            continue
        src = read_npz(path)
        if "time_bjd" not in src or "flux" not in src:
            raise ValueError(f"{path}: required columns are time_bjd and flux")
        t, f = src["time_bjd"], src["flux"]
        if len(t.shape) != 1 or f.shape != t.shape:
            raise ValueError(f"{path}: time_bjd and flux must be matching vectors")
        n = len(t)
        e = src.get("flux_err")
        if e is not None:
            if e.shape != t.shape:
                raise ValueError(f"{path}: flux_err must match time_bjd")
            if index == 0:
                err = []
            if err is None:
                raise ValueError("all input files must either provide flux_err or omit it")
            err.append(e.data)
        elif err is not None:
            raise ValueError("all input files must either provide flux_err or omit it")
        s = src.get("sector")
        if s is None:
            sectors = np.zeros(n, dtype=np.int64)
        elif len(s) == 1:
            sectors = np.full(n, int(s.data[0]), dtype=np.int64)
        elif len(s) == n:
            sectors = s.data.astype(np.int64)
        else:
            raise ValueError(f"{path}: sector must be a scalar or an observation vector")
        time.append(t.data)
        flux.append(f.data)
        group.append(np.array([label(index, int(x)) for x in sectors], dtype=np.int64))
    cat = lambda parts, dt=np.float64: np.concatenate(parts) if parts else np.zeros(0, dtype=dt)
    return Observations(cat(time), cat(flux), None if err is None else cat(err), cat(group, np.int64))
