"""The reference's on-disk formats, so the GPU path can load and write what the
Fortran host reads and writes: the grain microstructure file (file_media,
src/grain.f90:16-78: per layer file_grain, src/data.f90:219-320, then
file_field, src/field.f90:898-1008), the magnetostatic tensor cache
(file_tensor, src/tensor.f90:28-80, the mrm_N.dat files) and the
magnetisation file (file_mag, src/mag.f90:152-305; binary and Tecplot ASCII).

Binary files are Fortran unformatted sequential files as gfortran writes
them: each record framed by its byte length as a little-endian int32 before
and after it (a record over 2**31 - 9 bytes continues in subrecords whose
leading marker is negative); INTEGER is int32, LOGICAL int32 (1 true, 0
false), REAL(8) float64, REAL(4) float32; arrays in Fortran (column-major)
order.  Only the current layouts are written; reading the reference's "old"
grain and magnetisation layouts is not supported.
"""
from __future__ import annotations

import io
import struct
from typing import BinaryIO, Dict, List, Optional, Sequence, Tuple

import numpy as np

_MAX_SUB = 2 ** 31 - 9  # gfortran's largest subrecord


# ---------------------------------------------------------------------------
# Fortran sequential records
# ---------------------------------------------------------------------------

def write_record(f: BinaryIO, *items) -> None:
    """One record of the items in order (numpy arrays are written in Fortran
    order; Python ints as int32, floats as float64, bools as logical)."""
    parts = []
    for it in items:
        if isinstance(it, (bool, np.bool_)):
            parts.append(struct.pack("<i", 1 if it else 0))
        elif isinstance(it, (int, np.integer)):
            parts.append(struct.pack("<i", int(it)))
        elif isinstance(it, (float, np.floating)):
            parts.append(struct.pack("<d", float(it)))
        else:
            a = np.asarray(it)
            if a.dtype == np.bool_:
                a = a.astype("<i4")
            elif a.dtype.kind in "iu":
                a = a.astype("<i4")
            elif a.dtype == np.float32:
                a = a.astype("<f4")
            else:
                a = a.astype("<f8")
            parts.append(a.tobytes(order="F"))
    data = b"".join(parts)
    if len(data) > _MAX_SUB:
        raise NotImplementedError("records over 2 GiB (gfortran subrecords) are read, not written")
    n = struct.pack("<i", len(data))
    f.write(n + data + n)


def read_record(f: BinaryIO) -> bytes:
    """The bytes of the next record (joining subrecords); EOFError at the end."""
    out = []
    while True:
        head = f.read(4)
        if len(head) < 4:
            raise EOFError("end of file")
        (m,) = struct.unpack("<i", head)
        data = f.read(abs(m))
        tail = f.read(4)
        if len(data) != abs(m) or len(tail) != 4:
            raise ValueError("truncated record")
        out.append(data)
        if m >= 0:
            return b"".join(out)


class _Reader:
    """Sequential reads of typed items out of one record."""

    def __init__(self, data: bytes):
        self.b = memoryview(data)
        self.p = 0

    def ints(self, n: int = 1):
        a = np.frombuffer(self.b[self.p:self.p + 4 * n], dtype="<i4").astype(np.int64)
        self.p += 4 * n
        return a

    def int(self) -> int:
        return int(self.ints(1)[0])

    def logical(self) -> bool:
        return self.int() != 0

    def reals(self, n: int = 1, dtype="<f8"):
        size = np.dtype(dtype).itemsize
        a = np.frombuffer(self.b[self.p:self.p + size * n], dtype=dtype).astype(np.float64)
        self.p += size * n
        return a

    def real(self) -> float:
        return float(self.reals(1)[0])

    def done(self) -> bool:
        return self.p == len(self.b)


def _fortran(a: np.ndarray, shape: Tuple[int, ...]) -> np.ndarray:
    return np.asarray(a).reshape(shape, order="F")


# ---------------------------------------------------------------------------
# grain microstructure (file_media)
# ---------------------------------------------------------------------------

def write_grain_file(path: str, layers: Sequence[dict], nx: int, ny: int, dx: float, dy: float) -> None:
    """Writes file_media's records for every layer (data.f90:306-308, field.f90:977-996).

    Each layer dict: grid2grain (ny, nx) 1-based grain per cell (0: empty),
    grain2grid (ncell, 2) 1-based (i, j), grain2gridindex (N+1,), grain_area,
    ms, tc, tau (N,), hk (N, 2), and optional uni_axis (N, 3), cubic_axis
    (N, 3, 3) (row i = crystal axis i), and CSR tuples hx, lhx, uhx =
    (index (N+1,), grain (nnz,) 1-based, coef (nnz,))."""
    with open(path, "wb") as f:
        for il, L in enumerate(layers, start=1):
            g2g = np.asarray(L["grain2grid"], dtype=np.int64)
            n = len(L["ms"])
            write_record(f, nx, ny, il, float(dx), float(dy), n, len(g2g))
            write_record(f, np.asarray(L["grid2grain"]).T, g2g.T, np.asarray(L["grain2gridindex"]),
                         np.asarray(L["grain_area"], float))
            write_record(f, np.asarray(L["ms"], float), np.asarray(L["tc"], float), np.asarray(L["tau"], float))
            uni, cub = L.get("uni_axis"), L.get("cubic_axis")
            hx, lhx, uhx = L.get("hx"), L.get("lhx"), L.get("uhx")
            write_record(f, uni is not None, cub is not None, hx is not None, lhx is not None, uhx is not None,
                         np.asarray(L["hk"], float).T)
            if uni is not None:
                write_record(f, np.asarray(uni, float).T)
            if cub is not None:
                # cubic_axis(k, i, n): lab component k of crystal axis i
                write_record(f, np.transpose(np.asarray(cub, float), (2, 1, 0)))
            for csr in (hx, lhx, uhx):
                if csr is not None:
                    idx, gr, cf = (np.asarray(a) for a in csr)
                    write_record(f, idx, len(gr))
                    write_record(f, gr, np.asarray(cf, float))


def read_grain_file(path: str) -> Tuple[dict, List[dict]]:
    """Reads file_media's records (current layout) for every layer in the file.

    Returns ({nx, ny, dx, dy}, [layer dicts as write_grain_file takes])."""
    layers = []
    head = {}
    with open(path, "rb") as f:
        while True:
            try:
                r = _Reader(read_record(f))
            except EOFError:
                break
            nx, ny, il = r.int(), r.int(), r.int()
            dx, dy = r.real(), r.real()
            n, n2 = r.int(), r.int()
            head = dict(nx=nx, ny=ny, dx=dx, dy=dy)
            r = _Reader(read_record(f))
            L: Dict[str, object] = {"layer": il}
            L["grid2grain"] = _fortran(r.ints(nx * ny), (nx, ny)).T.copy()
            L["grain2grid"] = _fortran(r.ints(2 * n2), (2, n2)).T.copy()
            L["grain2gridindex"] = r.ints(n + 1)
            L["grain_area"] = r.reals(n)
            r = _Reader(read_record(f))
            L["ms"], L["tc"], L["tau"] = r.reals(n), r.reals(n), r.reals(n)
            r = _Reader(read_record(f))
            u_p, c_p, x_p, lx_p, ux_p = (r.logical() for _ in range(5))
            L["hk"] = _fortran(r.reals(2 * n), (2, n)).T.copy()
            L["uni_axis"] = _fortran(_Reader(read_record(f)).reals(3 * n), (3, n)).T.copy() if u_p else None
            if c_p:
                L["cubic_axis"] = np.transpose(_fortran(_Reader(read_record(f)).reals(9 * n), (3, 3, n)), (2, 1, 0)).copy()
            else:
                L["cubic_axis"] = None
            for key, on in (("hx", x_p), ("lhx", lx_p), ("uhx", ux_p)):
                if not on:
                    L[key] = None
                    continue
                r = _Reader(read_record(f))
                idx = r.ints(n + 1)
                nnz = r.int()
                r = _Reader(read_record(f))
                L[key] = (idx, r.ints(nnz), r.reals(nnz))
            layers.append(L)
    return head, layers


def grain_file_layers(medium, tc: float = 1e22, tau: float = 0.0) -> List[dict]:
    """Layer dicts of write_grain_file for a media.Medium (grain area from the
    cells each grain covers)."""
    out = []
    for lay in medium.layers:
        n = lay.N
        idx = np.asarray(lay.g2c_index)
        g2c = np.asarray(lay.g2c)
        grid = np.zeros((medium.ny, medium.nx), dtype=np.int64)
        for g in range(n):
            for q in range(idx[g], idx[g + 1]):
                grid[g2c[q, 1] - 1, g2c[q, 0] - 1] = g + 1
        cub = getattr(lay, "cubic_axis", None)
        out.append(dict(
            grid2grain=grid, grain2grid=g2c, grain2gridindex=idx,
            grain_area=np.diff(idx) * medium.dx * medium.dy,
            ms=np.asarray(lay.ms, float), tc=np.full(n, tc), tau=np.full(n, tau), hk=np.asarray(lay.hk, float),
            uni_axis=None if cub is not None else np.asarray(lay.axis, float), cubic_axis=cub,
            hx=None if lay.hx_index is None else (lay.hx_index, lay.hx_grain, lay.hx),
            lhx=lay.lhx, uhx=lay.uhx))
    return out


def medium_from_grain_file(path: str, dz: Sequence[float], *, il_space: Optional[Sequence[float]] = None,
                           alpha: float = 0.1, gamma: float = 1.76e7, floor_ms: float = 0.01,
                           boundary: int = 0):
    """A media.Medium from a grain file: grain volume = area x layer thickness,
    unit scales, m along +z, no applied field (set it on the layers)."""
    from . import media
    head, ls = read_grain_file(path)
    layers = []
    for k, L in enumerate(ls):
        n = len(L["ms"])
        uni = L["uni_axis"]
        lay = media.Layer(
            nx=head["nx"], ny=head["ny"], ms=L["ms"], vol=L["grain_area"] * dz[k],
            axis=uni if uni is not None else np.zeros((n, 3)), hk=L["hk"],
            hk_scale=np.ones(n), ms_scale=np.ones(n), alpha_scale=np.ones(n), alpha=alpha, gamma=gamma,
            floor_ms=floor_ms, g2c_index=L["grain2gridindex"].astype(np.int32),
            g2c=L["grain2grid"].astype(np.int32),
            hx_index=None if L["hx"] is None else L["hx"][0].astype(np.int32),
            hx_grain=None if L["hx"] is None else L["hx"][1].astype(np.int32),
            hx=None if L["hx"] is None else L["hx"][2],
            uhx=None if L["uhx"] is None else tuple(np.asarray(a) for a in L["uhx"]),
            lhx=None if L["lhx"] is None else tuple(np.asarray(a) for a in L["lhx"]))
        lay.cubic_axis = L["cubic_axis"]
        layers.append(lay)
    m0 = [np.tile([0.0, 0.0, 1.0], (lay.N, 1)) for lay in layers]
    return media.Medium(nx=head["nx"], ny=head["ny"], dx=head["dx"], dy=head["dy"], dz=list(dz),
                        il_space=list(il_space) if il_space is not None else [0.0] * len(layers),
                        layers=layers, boundary=boundary, m0=m0)


# ---------------------------------------------------------------------------
# magnetostatic tensor cache (file_tensor)
# ---------------------------------------------------------------------------

def write_tensor_cache(path: str, n2d: np.ndarray, *, nx: int, ny: int, imx: int, imy: int, dx: float, dy: float,
                       dz: Sequence[float], il_space: Sequence[float], head: bool = False, sul: bool = False,
                       head_mu: float = 1.0, sul_mu: float = 1.0, fly_height: float = 0.0,
                       space_to_sul: float = 0.0) -> None:
    """n2d as numpy (n_lay, n_lay, 9, ny, nx) = the reference's n2d(nx, ny, 9, n_lay, n_lay)."""
    nl = len(dz)
    a = np.asarray(n2d, float)
    if a.shape != (nl, nl, 9, ny, nx):
        raise ValueError(f"n2d must be ({nl}, {nl}, 9, {ny}, {nx})")
    with open(path, "wb") as f:
        write_record(f, bool(head), bool(sul), nx, ny, nl, imx, imy, float(dx), float(dy), float(head_mu),
                     float(sul_mu), float(fly_height), float(space_to_sul), np.asarray(dz, float),
                     np.asarray(il_space, float))
        data = np.ascontiguousarray(a)
        # C order (nl, nl, 9, ny, nx) is the Fortran order of (nx, ny, 9, nl, nl)
        rec = data.tobytes(order="C")
        n = struct.pack("<i", len(rec))
        if len(rec) > _MAX_SUB:
            raise NotImplementedError("tensor records over 2 GiB")
        f.write(n + rec + n)


def read_tensor_cache(path: str) -> Tuple[dict, np.ndarray]:
    """(header, n2d as numpy (n_lay, n_lay, 9, ny, nx)) of an mrm_N.dat file."""
    with open(path, "rb") as f:
        r = _Reader(read_record(f))
        h = dict(head=r.logical(), sul=r.logical(), nx=r.int(), ny=r.int(), n_lay=r.int(), imx=r.int(),
                 imy=r.int(), dx=r.real(), dy=r.real(), head_mu=r.real(), sul_mu=r.real(), fly_height=r.real(),
                 space_to_sul=r.real())
        h["dz"] = r.reals(h["n_lay"])
        h["il_space"] = r.reals(h["n_lay"])
        data = read_record(f)
    nl, nx, ny = h["n_lay"], h["nx"], h["ny"]
    n2d = np.frombuffer(data, dtype="<f8").reshape((nl, nl, 9, ny, nx)).copy()
    return h, n2d


# ---------------------------------------------------------------------------
# magnetisation (file_mag)
# ---------------------------------------------------------------------------

def write_mag(path: str, m_layers: Sequence[np.ndarray], ms_layers: Sequence[np.ndarray], nx: int, ny: int,
              ms_nom: Sequence[float]) -> None:
    """Binary magnetisation (mag.f90:290-295): per layer (nx, ny, N, ms_nom),
    then m * Ms per grain as (3, N)."""
    with open(path, "wb") as f:
        for m, ms, nom in zip(m_layers, ms_layers, ms_nom):
            m = np.asarray(m, float)
            write_record(f, nx, ny, len(m), float(nom))
            write_record(f, (m * np.asarray(ms, float)[:, None]).T)


def read_mag(path: str, n_layers: int) -> List[dict]:
    """Binary magnetisation: per layer {nx, ny, ms_nom, m (N, 3) unit, ms_file
    (N,) the stored magnitudes} (mag.f90:232-250 normalises m; the reference
    then rescales Ms by ms_nom / stored ms_nom, which is left to the caller)."""
    out = []
    with open(path, "rb") as f:
        for _ in range(n_layers):
            r = _Reader(read_record(f))
            nx, ny, n = r.int(), r.int(), r.int()
            nom = r.real()
            mm = _fortran(_Reader(read_record(f)).reals(3 * n), (3, n)).T.copy()
            mag = np.linalg.norm(mm, axis=1)
            m = np.where(mag[:, None] > 0, mm / np.where(mag > 0, mag, 1.0)[:, None], 0.0)
            out.append(dict(nx=nx, ny=ny, ms_nom=nom, m=m, ms_file=mag))
    return out


def write_mag_ascii(path: str, m_layers: Sequence[np.ndarray], ms_layers: Sequence[np.ndarray],
                    ms_scale_layers: Sequence[np.ndarray], grid2grain_layers: Sequence[np.ndarray], nx: int,
                    ny: int, zone_t: float = 0.0) -> None:
    """Tecplot ASCII magnetisation (mag.f90:266-279): a ZONE line per layer,
    then per cell (i, j, layer) and m * Ms * ms_scale of its grain (0 if empty)."""
    with open(path, "w") as f:
        for k, (m, ms, mss, grid) in enumerate(zip(m_layers, ms_layers, ms_scale_layers, grid2grain_layers), 1):
            f.write(f'ZONE T="{zone_t:9.2f}", I={nx:5d}, J={ny:5d}, K={1:3d} F=POINT\n')
            for j in range(ny):
                for i in range(nx):
                    g = int(grid[j, i])
                    v = np.asarray(m[g - 1], float) * ms[g - 1] * mss[g - 1] if g > 0 else np.zeros(3)
                    f.write(f"{i + 1:5d}{j + 1:5d}{k:5d}" + "".join(f" {x:12.5E}" for x in v) + "\n")


def read_mag_ascii(path: str, grid2grain_layers: Sequence[np.ndarray], n_grains: Sequence[int]) -> List[np.ndarray]:
    """Tecplot ASCII magnetisation (mag.f90:196-211): each grain takes the unit
    vector of the (last) cell listed for it; grains without a cell stay zero."""
    out = []
    with open(path) as f:
        lines = f.read().splitlines()
    p = 0
    for grid, n in zip(grid2grain_layers, n_grains):
        head = lines[p]
        nx, ny = int(head[22:27]), int(head[31:36])
        p += 1
        m = np.zeros((n, 3))
        for j in range(ny):
            for i in range(nx):
                ln = lines[p]
                p += 1
                v = np.array([float(ln[15 + 13 * q + 1:15 + 13 * (q + 1)]) for q in range(3)])
                g = int(grid[j, i])
                if g > 0:
                    mg = float(v @ v)
                    m[g - 1] = v / np.sqrt(mg) if mg != 0.0 else v
        out.append(m)
    return out


# ---------------------------------------------------------------------------
# Tabulated applied-field files (file_applied, applied.f90:711-813)
# ---------------------------------------------------------------------------

def _tecplot_size(line: str) -> Tuple[int, int]:
    """I= and J= of a Tecplot zone line, as file_applied reads them (the digits
    after 'I='/'i=' and 'J='/'j=')."""
    def after(keys):
        for k in keys:
            p = line.find(k)
            if p >= 0:
                q = p + 2
                while q < len(line) and line[q] == " ":
                    q += 1
                r = q
                while r < len(line) and line[r].isdigit():
                    r += 1
                return int(line[q:r])
        raise ValueError(f"no {keys[0]} in {line!r}")
    return after(("I=", "i=")), after(("J=", "j="))


def _is_data_line(line: str) -> bool:
    """file_applied's test for the first data line: nothing but blanks, digits,
    signs, points and exponent letters."""
    s = line.strip()
    return len(s) > 0 and all(c in " 0123456789+-.eEdD" for c in s)


def read_field_file(path: str, nval: int = 3, scale: float = 1.0):
    """A tabulated field (nval 3) or temperature (nval 1) profile as file_applied
    reads it: the zone line with I= and J= gives the node counts, the data start
    at the first purely numeric line, then one list-directed record per node,
    x fastest.  Vector records are FEM coordinates `x y z Hx Hy Hz`, mapped to
    the model's axes (x -> -x, z -> y, H_y <-> H_z, H_x -> -H_x) with the x nodes
    reversed so they ascend; the values are multiplied by `scale`.  Returns
    (xpos (nx,), ypos (ny,), values (ny, nx, 3) or (ny, nx))."""
    with open(path) as f:
        lines = f.read().splitlines()
    p = 0
    while p < len(lines) and not any(k in lines[p] for k in ("I=", "i=", "J=", "j=")):
        p += 1
    if p == len(lines):
        raise ValueError("no Tecplot zone line (I=, J=)")
    nx, ny = _tecplot_size(lines[p].strip())
    p += 1
    while p < len(lines) and not _is_data_line(lines[p]):
        p += 1
    tokens: List[str] = []

    def record(k: int) -> List[float]:
        # a list-directed read starts at a new record and continues onto the
        # following ones until it has its k values; the rest of the last one is skipped
        nonlocal p
        vals: List[float] = []
        while len(vals) < k:
            if p >= len(lines):
                raise ValueError("field file ends early")
            vals += [float(t.replace("d", "e").replace("D", "e")) for t in lines[p].replace(",", " ").split()]
            p += 1
        return vals[:k]

    xpos, ypos = np.zeros(nx), np.zeros(ny)
    vals = np.zeros((ny, nx, 3)) if nval != 1 else np.zeros((ny, nx))
    for j in range(ny):
        for i in range(nx):
            if nval == 1:
                x, y, v = record(3)
                xpos[i], ypos[j], vals[j, i] = x, y, v
            else:
                x, _, y, h1, h3, h2 = record(6)
                ii = nx - 1 - i
                xpos[ii], ypos[j] = x, y
                vals[j, ii] = (h1, h2, h3)
    if nval != 1:
        xpos = -xpos
        vals[..., 0] = -vals[..., 0]
    if scale != 1.0:
        vals = vals * scale
    return xpos, ypos, vals


def write_field_file(path: str, xpos: np.ndarray, ypos: np.ndarray, vfld: np.ndarray,
                     title: str = "write field") -> None:
    """Writes a vector profile (ny, nx, 3) on ascending nodes in the FEM
    orientation that read_field_file (file_applied) maps back."""
    xpos, ypos, vfld = np.asarray(xpos, float), np.asarray(ypos, float), np.asarray(vfld, float)
    nx, ny = xpos.size, ypos.size
    with open(path, "w") as f:
        f.write(f'TITLE = "{title}"\n')
        f.write('VARIABLES = "x" "y" "z" "Hx" "Hy" "Hz"\n')
        f.write(f"ZONE I={nx}, J={ny}, F=POINT\n")
        for j in range(ny):
            for i in range(nx):
                ii = nx - 1 - i  # the file's i-th node is the model's node nx-1-i, at -x
                h = vfld[j, ii]
                f.write(f"{-xpos[ii]:.17e} {0.0:.17e} {ypos[j]:.17e} {-h[0]:.17e} {h[2]:.17e} {h[1]:.17e}\n")
