"""spiffe input decks on libspiffe_b200 (binding of spiffe_b200_session.h).

    python -m spiffe_b200.session deck.spiffe [--precision f64|split32]

runs a spiffe input file the way ``spiffe deck.spiffe`` does (spiffe.c:92-365):
define_geometry, define_cathode, define_solenoid, define_antenna,
define_screen, define_test_beam, set_constant_fields, poisson_correction,
load_fields, define_field_saving and integrate are executed by the library's
command session (C++, spiffe_b200/csrc/session.cu); the integration runs on
the GPU.  Screens and field saves are written as SDDS files.

``Session`` is the same from Python, with the problem's arrays and the
device instance open for inspection.  ``read_sdds`` reads the SDDS files the
session writes (and the ASCII/binary SDDS tables spiffe reads).
"""
from __future__ import annotations

import argparse
import ctypes as C
import struct
import sys

import numpy as np

from . import abi, gpu

SETTINGS = ("verbose", "deposit_order", "particle_capacity", "screen_capacity", "flush_steps", "compaction",
            "screen_momentum", "poisson_solver")


class Session:
    """A spiffe command session; state persists across execute() calls."""

    def __init__(self, precision="f64", rootname=None, **settings):
        self.lib = gpu.load()
        self.precision = gpu.PRECISION_SPLIT32 if precision == "split32" else gpu.PRECISION_F64
        h = C.c_void_p()
        self._check(self.lib.spiffe_session_create(self.precision, rootname.encode() if rootname else None,
                                                   C.byref(h)))
        self.h = h
        for k, v in settings.items():
            self.set(k, v)

    def _check(self, rc):
        if rc < 0:
            raise gpu.SpiffeGpuError(f"spiffe session error {rc}: {self.lib.spiffe_gpu_last_error().decode()}")
        return rc

    def set(self, name, value):
        if name not in SETTINGS:
            raise KeyError(name)
        self._check(self.lib.spiffe_session_set(self.h, name.encode(), float(value)))

    def execute(self, text):
        """Runs namelist commands; returns 1 after &stop, else 0."""
        return self._check(self.lib.spiffe_session_execute(self.h, text.encode()))

    def run_file(self, path):
        return self._check(self.lib.spiffe_session_run_file(self.h, str(path).encode()))

    def mesh(self):
        m = abi.Mesh()
        self._check(self.lib.spiffe_session_mesh(self.h, C.byref(m)))
        return m

    def fields(self):
        """abi.Fields holding the session's current arrays (from the device after an integrate)."""
        m = self.mesh()
        f = abi.Fields(m.nz, m.nr, m.zmin, m.zmax, m.rmax, modes=m.modes, left_bc=m.left_bc, right_bc=m.right_bc,
                       lower_bc=m.lower_bc, upper_bc=m.upper_bc)
        f.mesh = m
        for n in ("EzImposed", "ErImposed", "PsiImposed", "Psi", "Q", "Jz"):
            f.a.setdefault(n, np.zeros(f.shape))
        if m.has_solenoid:
            f.a["BzImposed"] = np.zeros(f.shape)
            f.a["BrImposed"] = np.zeros(f.shape)
        s = f.c()
        self._check(self.lib.spiffe_session_fields(self.h, C.byref(s)))
        return f

    def instance(self):
        """gpu.GpuInstance view of the device problem (None before integrate)."""
        h = C.c_void_p()
        self._check(self.lib.spiffe_session_instance(self.h, C.byref(h)))
        return gpu.GpuInstance.attach(h, self.precision) if h.value else None

    def steps(self):
        return self.lib.spiffe_session_steps(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.spiffe_session_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solenoid_field(fields, radius, z_start, z_end, current=0.0, Bz_peak=0.0, turns=1, symmetry=0,
                   evaluation_radius_limit=0.0, bucking=0, z_buck=0.0):
    """Adds define_solenoid's ring-coil field to fields['BzImposed'/'BrImposed']
    (created if absent); returns the current applied."""
    lib = gpu.load()
    for n in ("BzImposed", "BrImposed"):
        if n not in fields.a:
            fields.a[n] = np.zeros(fields.shape)
    o = abi.SolenoidOptions(radius, evaluation_radius_limit, z_start, z_end, current, Bz_peak, turns, symmetry,
                            bucking, z_buck)
    cur = C.c_double()
    rc = lib.spiffe_solenoid_add(C.byref(fields.mesh), C.byref(o), fields["BzImposed"].ctypes.data_as(abi.D),
                                 fields["BrImposed"].ctypes.data_as(abi.D), C.byref(cur))
    if rc < 0:
        raise gpu.SpiffeGpuError(lib.spiffe_gpu_last_error().decode())
    fields.mesh.has_solenoid = 1
    return cur.value


# ----------------------------------------------------------------- SDDS files

_SDDS_TYPES = {"double": "d", "float": "f", "long64": "q", "ulong64": "Q", "long": "i", "ulong": "I",
               "short": "h", "ushort": "H", "character": "c", "string": None}


def _namelists(header):
    from shlex import shlex

    out = []
    for line in header:
        line = line.strip()
        if not line.startswith("&"):
            continue
        group = line[1:].split()[0]
        body = line[len(group) + 1:].replace("&end", "")
        lex = shlex(body, posix=True)
        lex.whitespace += ","
        lex.wordchars += ".-+$/%*#:;()[]{}<>^!|~'@?"
        toks = list(lex)
        d = {}
        i = 0
        while i < len(toks):
            if i + 2 < len(toks) and toks[i + 1] == "=":
                d[toks[i].lower()] = toks[i + 2]
                i += 3
            elif "=" in toks[i]:
                k, v = toks[i].split("=", 1)
                d[k.lower()] = v
                i += 1
            else:
                i += 1
        out.append((group, d))
    return out


def read_sdds(path):
    """Pages of an SDDS1 file as a list of dicts: {"parameters": {...},
    "columns": {name: numpy array}} (binary or ASCII; no arrays)."""
    raw = open(path, "rb").read()
    if not raw.startswith(b"SDDS"):
        raise ValueError(f"{path} is not an SDDS file")
    pos = raw.index(b"\n") + 1
    header, big = [], False
    while True:
        eol = raw.index(b"\n", pos)
        line = raw[pos:eol].decode("latin-1")
        pos = eol + 1
        if line.startswith("!"):
            big = big or "big-endian" in line
            continue
        header.append(line)
        if line.strip().startswith("&data"):
            break
    nl = _namelists(header)
    params = [d for g, d in nl if g == "parameter"]
    cols = [d for g, d in nl if g == "column"]
    data = [d for g, d in nl if g == "data"][0]
    pages = []
    if data.get("mode", "ascii") == "binary":
        end = ">" if big else "<"
        cm = int(data.get("column_major_order", "0"))
        while pos + 4 <= len(raw):
            (rows,) = struct.unpack_from(end + "i", raw, pos)
            pos += 4
            page = {"parameters": {}, "columns": {}}
            for p in params:
                if "fixed_value" in p:
                    page["parameters"][p["name"]] = p["fixed_value"]
                    continue
                t = p["type"]
                if t == "string":
                    (n,) = struct.unpack_from(end + "i", raw, pos)
                    page["parameters"][p["name"]] = raw[pos + 4:pos + 4 + n].decode()
                    pos += 4 + n
                elif t == "character":
                    page["parameters"][p["name"]] = raw[pos:pos + 1].decode()
                    pos += 1
                else:
                    (v,) = struct.unpack_from(end + _SDDS_TYPES[t], raw, pos)
                    page["parameters"][p["name"]] = v
                    pos += struct.calcsize(_SDDS_TYPES[t])
            if any(c["type"] == "string" for c in cols):
                raise ValueError("string columns are not supported")
            dt = np.dtype([(c["name"], end + _SDDS_TYPES[c["type"]]) for c in cols])
            if cm:
                for c in cols:
                    t = np.dtype(end + _SDDS_TYPES[c["type"]])
                    page["columns"][c["name"]] = np.frombuffer(raw, t, rows, pos).copy()
                    pos += rows * t.itemsize
            else:
                rec = np.frombuffer(raw, dt, rows, pos)
                pos += rows * dt.itemsize
                for c in cols:
                    page["columns"][c["name"]] = rec[c["name"]].copy()
            pages.append(page)
    else:
        lines = [ln for ln in raw[pos:].decode("latin-1").splitlines() if not ln.lstrip().startswith("!")]
        no_counts = int(data.get("no_row_counts", "0"))
        i = 0
        while i < len(lines):
            while i < len(lines) and not lines[i].strip():
                i += 1
            if i >= len(lines):
                break
            page = {"parameters": {}, "columns": {}}
            for p in params:
                if "fixed_value" in p:
                    page["parameters"][p["name"]] = p["fixed_value"]
                else:
                    page["parameters"][p["name"]] = lines[i].strip()
                    i += 1
            rows = []
            if no_counts:
                while i < len(lines) and lines[i].strip():
                    rows.append(lines[i].split())
                    i += 1
            else:
                n = int(lines[i])
                i += 1
                for _ in range(n):
                    rows.append(lines[i].split())
                    i += 1
            for k, c in enumerate(cols):
                page["columns"][c["name"]] = np.array([float(r[k]) for r in rows])
            pages.append(page)
    return pages


def write_sdds_ascii(path, columns, parameters=None):
    """A one-page ASCII SDDS table of double columns (waveforms, profiles)."""
    with open(path, "w") as f:
        f.write("SDDS1\n")
        for k in parameters or {}:
            f.write(f"&parameter name={k}, type=double, &end\n")
        for k in columns:
            f.write(f"&column name={k}, type=double, &end\n")
        f.write("&data mode=ascii, &end\n")
        for v in (parameters or {}).values():
            f.write(f"{v!r}\n")
        cols = [np.asarray(v, np.float64) for v in columns.values()]
        f.write(f"{len(cols[0])}\n")
        for row in zip(*cols):
            f.write(" ".join(repr(float(x)) for x in row) + "\n")


def write_field_save(path, fields, times):
    """A field-save file (the layout of save_fields, field_saving.c:67-119)
    from abi.Fields: one binary page per entry of `times`, each holding the
    same arrays.  load_fields reads it."""
    m = fields.mesh
    tm, te = bool(m.modes & abi.FL_TM_FIELDS), bool(m.modes & abi.FL_TE_FIELDS)
    hdr = ["SDDS1", "!# little-endian", '&description contents="spiffe field saves", &end',
           '&parameter name=time, units=s, description="time of field save", type=double, &end',
           '&parameter name=version, description="save version", type=long, fixed_value=4, &end',
           f'&parameter name=nr, description="number of r grid lines", type=long, fixed_value={m.nr}, &end',
           f'&parameter name=nz, description="number of z grid lines", type=long, fixed_value={m.nz}, &end',
           f'&parameter name=dr, units=m, description="spacing of r grid lines", type=double, '
           f'fixed_value={m.dr!r}, &end',
           f'&parameter name=dz, units=m, description="spacing of z grid lines", type=double, '
           f'fixed_value={m.dz!r}, &end']
    for k in ("zmin", "zmax", "rmax"):
        hdr.append(f"&parameter name={k}, units=m, type=double, fixed_value={getattr(m, k)!r}, &end")
    hdr.append("&parameter name=zt, units=m, type=double, fixed_value=0, &end")
    hdr.append(f"&parameter name=TMfields, type=character, fixed_value={'y' if tm else 'n'}, &end")
    hdr.append(f"&parameter name=TEfields, type=character, fixed_value={'y' if te else 'n'}, &end")
    hdr.append("&column name=metalFlags, type=long, &end")
    names = (["Ez", "Er", "Jz", "Jr", "Bphi", "Bphi2"] if tm else []) + \
            (["Ephi", "Jphi", "Br", "Br2", "Bz", "Bz2"] if te else [])
    units = {"E": "V/m", "J": "A/m$a2$n", "B": "T"}
    for n in names:
        hdr.append(f"&column name={n}, units={units[n[0]]}, type=double, &end")
    hdr.append("&data mode=binary, &end")
    dt = np.dtype([("metalFlags", "<i4")] + [(n, "<f8") for n in names])
    rec = np.zeros(fields.flags.size, dt)
    for n in names:
        rec[n] = fields[n].ravel()
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode())
        for t in times:
            f.write(struct.pack("<i", rec.size) + struct.pack("<d", t))
            f.write(rec.tobytes())


def main(argv=None):
    ap = argparse.ArgumentParser(description="Run a spiffe input file on the GPU.")
    ap.add_argument("inputfile")
    ap.add_argument("--precision", choices=("f64", "split32"), default="f64")
    ap.add_argument("--quiet", action="store_true")
    a = ap.parse_args(argv)
    root = a.inputfile.rsplit("/", 1)[-1].split(".")[0]
    with Session(a.precision, rootname=root, verbose=0 if a.quiet else 1) as s:
        try:
            rc = s.run_file(a.inputfile)
        except gpu.SpiffeGpuError as e:
            print(e, file=sys.stderr)
            return 1
    return 1 if rc == 1 else 0


if __name__ == "__main__":
    sys.exit(main())
