"""OIFITS tables and a reader for OIFITS files (FITS binary tables).

The reference reads OIFITS through cfitsio (gpair1/trunk/read_fits.c:228-603,
structs in gpair1/trunk/exchange.h:63-141). This module holds the same tables
as numpy arrays:

* :class:`WavelengthTable` -- OI_WAVELENGTH (EFF_WAVE, EFF_BAND as float32, metres)
* :class:`Vis2Table`       -- OI_VIS2 (per row: TARGET_ID, UCOORD, VCOORD; per row and
  channel: VIS2DATA, VIS2ERR, FLAG)
* :class:`T3Table`         -- OI_T3 (per row: TARGET_ID, U1/V1/U2/V2COORD; per row and
  channel: T3AMP, T3AMPERR, T3PHI, T3PHIERR, FLAG)

:func:`read_oifits` parses a FITS file with a small reader written for this
project from the public FITS standard (2880-byte blocks, 80-character header
cards, big-endian binary-table rows). Column types L, A, I, J, E, D are
supported, which covers the OIFITS tables.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List

import numpy as np


@dataclass
class WavelengthTable:
    insname: str
    eff_wave: np.ndarray  # float32 [nwave], metres
    eff_band: np.ndarray  # float32 [nwave], metres


@dataclass
class Vis2Table:
    insname: str
    target_id: np.ndarray  # int32 [nrec]
    ucoord: np.ndarray  # float64 [nrec], metres
    vcoord: np.ndarray  # float64 [nrec]
    vis2data: np.ndarray  # float64 [nrec, nwave]
    vis2err: np.ndarray  # float64 [nrec, nwave]
    flag: np.ndarray  # uint8 [nrec, nwave]

    @property
    def nwave(self) -> int:
        return self.vis2data.shape[1]


@dataclass
class T3Table:
    insname: str
    target_id: np.ndarray
    u1coord: np.ndarray
    v1coord: np.ndarray
    u2coord: np.ndarray
    v2coord: np.ndarray
    t3amp: np.ndarray  # float64 [nrec, nwave]; NaN = amplitude not measured
    t3amperr: np.ndarray
    t3phi: np.ndarray  # degrees
    t3phierr: np.ndarray
    flag: np.ndarray

    @property
    def nwave(self) -> int:
        return self.t3amp.shape[1]


@dataclass
class OIFits:
    """An OIFITS data set: tables in file order (HDU order matters to the matcher)."""

    wavelengths: List[WavelengthTable] = field(default_factory=list)
    vis2: List[Vis2Table] = field(default_factory=list)
    t3: List[T3Table] = field(default_factory=list)
    target_id: int = 1

    def wavelength(self, insname: str) -> WavelengthTable:
        for w in self.wavelengths:
            if w.insname == insname:
                return w
        raise KeyError(f"no OI_WAVELENGTH table for INSNAME {insname!r}")

    @property
    def num_vis2(self) -> int:
        return int(sum(t.vis2data.size for t in self.vis2))

    @property
    def num_t3(self) -> int:
        return int(sum(t.t3amp.size for t in self.t3))


# ----------------------------------------------------------------- FITS reader

_BLOCK = 2880
_TFORM_DTYPE = {"L": ("S1", 1), "A": ("S1", 1), "I": (">i2", 2), "J": (">i4", 4), "K": (">i8", 8),
                "E": (">f4", 4), "D": (">f8", 8), "B": ("u1", 1)}


def _parse_header(buf: bytes, pos: int):
    cards: Dict[str, str] = {}
    order = []
    while True:
        block = buf[pos:pos + _BLOCK]
        if len(block) < _BLOCK:
            raise ValueError("truncated FITS header")
        pos += _BLOCK
        done = False
        for i in range(0, _BLOCK, 80):
            card = block[i:i + 80].decode("ascii", "replace")
            key = card[:8].strip()
            if key == "END":
                done = True
                break
            if card[8:10] == "= ":
                val = card[10:]
                if val.lstrip().startswith("'"):
                    s = val.lstrip()[1:]
                    end = s.find("'")
                    while end >= 0 and end + 1 < len(s) and s[end + 1] == "'":
                        end = s.find("'", end + 2)
                    val = s[:end].rstrip()
                else:
                    val = val.split("/")[0].strip()
                cards[key] = val
                order.append(key)
        if done:
            return cards, pos


def _parse_tform(tform: str):
    tform = tform.strip()
    i = 0
    while i < len(tform) and tform[i].isdigit():
        i += 1
    repeat = int(tform[:i]) if i else 1
    code = tform[i]
    return repeat, code


def _read_bintable(buf: bytes, pos: int, cards: Dict[str, str]):
    naxis1 = int(cards["NAXIS1"])
    naxis2 = int(cards["NAXIS2"])
    tfields = int(cards["TFIELDS"])
    cols = {}
    offset = 0
    raw = np.frombuffer(buf, dtype=np.uint8, count=naxis1 * naxis2, offset=pos).reshape(naxis2, naxis1)
    for c in range(1, tfields + 1):
        name = cards.get(f"TTYPE{c}", f"COL{c}").strip().upper()
        repeat, code = _parse_tform(cards[f"TFORM{c}"])
        dt, size = _TFORM_DTYPE[code]
        nbytes = repeat * size
        chunk = np.ascontiguousarray(raw[:, offset:offset + nbytes])
        if code == "A":
            cols[name] = [bytes(r).decode("ascii", "replace").rstrip("\x00 ") for r in chunk]
        elif code == "L":
            cols[name] = (chunk == ord("T")).astype(np.uint8).reshape(naxis2, repeat)
        else:
            arr = chunk.view(dt).reshape(naxis2, repeat).astype(dt.replace(">", "="))
            cols[name] = arr
        offset += nbytes
    heap = int(cards.get("PCOUNT", "0"))
    size = naxis1 * naxis2 + heap
    return cols, pos + ((size + _BLOCK - 1) // _BLOCK) * _BLOCK


def read_oifits(path: str, target_id: int | None = None) -> OIFits:
    """Parse OI_WAVELENGTH, OI_VIS2 and OI_T3 tables from an OIFITS file."""
    with open(path, "rb") as f:
        buf = f.read()
    out = OIFits()
    pos = 0
    first_target = None
    while pos < len(buf):
        cards, pos = _parse_header(buf, pos)
        if cards.get("XTENSION", "").strip() != "BINTABLE":
            naxis = int(cards.get("NAXIS", "0"))
            size = 0
            if naxis:
                size = abs(int(cards["BITPIX"])) // 8
                for a in range(1, naxis + 1):
                    size *= int(cards[f"NAXIS{a}"])
            pos += ((size + _BLOCK - 1) // _BLOCK) * _BLOCK
            continue
        cols, pos = _read_bintable(buf, pos, cards)
        ext = cards.get("EXTNAME", "").strip()
        ins = cards.get("INSNAME", "").strip()
        if ext == "OI_TARGET" and first_target is None:
            first_target = int(np.asarray(cols["TARGET_ID"]).ravel()[0])
        elif ext == "OI_WAVELENGTH":
            out.wavelengths.append(WavelengthTable(ins, cols["EFF_WAVE"][:, 0].astype(np.float32),
                                                   cols["EFF_BAND"][:, 0].astype(np.float32)))
        elif ext == "OI_VIS2":
            out.vis2.append(Vis2Table(
                ins, cols["TARGET_ID"][:, 0].astype(np.int32), cols["UCOORD"][:, 0].astype(np.float64),
                cols["VCOORD"][:, 0].astype(np.float64), cols["VIS2DATA"].astype(np.float64),
                cols["VIS2ERR"].astype(np.float64), cols["FLAG"].astype(np.uint8)))
        elif ext == "OI_T3":
            out.t3.append(T3Table(
                ins, cols["TARGET_ID"][:, 0].astype(np.int32),
                cols["U1COORD"][:, 0].astype(np.float64), cols["V1COORD"][:, 0].astype(np.float64),
                cols["U2COORD"][:, 0].astype(np.float64), cols["V2COORD"][:, 0].astype(np.float64),
                cols["T3AMP"].astype(np.float64), cols["T3AMPERR"].astype(np.float64),
                cols["T3PHI"].astype(np.float64), cols["T3PHIERR"].astype(np.float64),
                cols["FLAG"].astype(np.uint8)))
    out.target_id = target_id if target_id is not None else (first_target if first_target is not None else 1)
    return out


# ------------------------------------------------------------ FITS images

def read_fits_image(path: str):
    """Primary-HDU image of a FITS file as float32 [NAXIS2][NAXIS1] (x fastest), plus its header cards."""
    with open(path, "rb") as f:
        buf = f.read()
    cards, pos = _parse_header(buf, 0)
    bitpix = int(cards["BITPIX"])
    naxis = int(cards.get("NAXIS", "0"))
    if naxis != 2:
        raise ValueError(f"{path}: expected a 2-D primary image, NAXIS = {naxis}")
    nx, ny = int(cards["NAXIS1"]), int(cards["NAXIS2"])
    dt = {8: "u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}[bitpix]
    data = np.frombuffer(buf, dtype=dt, count=nx * ny, offset=pos).reshape(ny, nx).astype(np.float64)
    data = data * float(cards.get("BSCALE", "1")) + float(cards.get("BZERO", "0"))
    return data.astype(np.float32), cards


def _card(key: str, value) -> bytes:
    if isinstance(value, bool):
        v = "T" if value else "F"
        s = f"{key:<8}= {v:>20}"
    elif isinstance(value, (int, np.integer)):
        s = f"{key:<8}= {int(value):>20}"
    elif isinstance(value, (float, np.floating)):
        s = f"{key:<8}= {float(value):>20.12G}"
    else:
        text = str(value).replace("'", "''")
        s = f"{key:<8}= '{text:<8}'"
    return s[:80].ljust(80).encode("ascii")


def write_fits_image(path: str, image: np.ndarray, cards: Dict[str, object] | None = None):
    """Write a float32 image [ny][nx] as a FITS primary HDU (BITPIX -32, big-endian)."""
    img = np.asarray(image, np.float32)
    if img.ndim != 2:
        raise ValueError("image must be 2-D")
    head = [_card("SIMPLE", True), _card("BITPIX", -32), _card("NAXIS", 2), _card("NAXIS1", img.shape[1]),
            _card("NAXIS2", img.shape[0])]
    for k, v in (cards or {}).items():
        head.append(_card(k.upper()[:8], v))
    head.append(b"END".ljust(80))
    hdr = b"".join(head)
    hdr += b" " * ((-len(hdr)) % _BLOCK)
    data = img.astype(">f4").tobytes()
    data += b"\0" * ((-len(data)) % _BLOCK)
    with open(path, "wb") as f:
        f.write(hdr + data)
