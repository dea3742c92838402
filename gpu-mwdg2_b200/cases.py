"""Seeded synthetic inputs in the reference's file formats.

Writes `.par`, ESRI-ASCII `.dem`/`.start`, `.bci`, `.bdy` and `.stage` files in the
dialect the reference reads (keyword readers `input/read_keyword_*.cpp`, raster reader
`input/read_raster_file.cpp:26-46`, boundary/point-source readers
`classes/Boundary.h`, `classes/PointSources.h:251-279`, time series
`classes/Boundary.h:427-466`, stage points `classes/StagePoints.h:124-137`).

The same files feed this library, the CPU oracle and the reference build, so every
implementation sees byte-identical inputs. Generators:

* circular_dam_break  - flat bed, closed walls, radial depth step (256^2 parity case).
* fbm_catchment       - fractional-Brownian-motion DEM, dry start, west-edge point
                        inflow with a triangular hydrograph (4096^2 benchmark case).
* lake_at_rest        - still water over an fBm bed (well-balancing checks).
* ensemble            - seeded mix of fBm catchments with dam breaks or point inflows
                        of uneven sizes (batched-ensemble benchmark).
* urban_catchment     - fBm base with axis-aligned building blocks, a lake at rest and a
                        rising west-edge point inflow (8192^2 urban benchmark case).
* bc_edges            - a lake over an fBm bed with boundary segments of every type
                        (FREE, HFIX, HVAR, QFIX, QVAR) on the four sides.
* start_q_nodata      - a DEM narrower than the mesh with -9999 (no-data) cells, and an
                        initial discharge read from .start.Qx/.Qy rasters (startq2d).

Reference quirks the generators respect (they would otherwise change the physics):
* `wall_height` is set above every bed value, because `operators/dg2_update.cu:46`
  skips cells whose bed equals `wall_height` (a flat bed with wall_height 0 would
  never update).
* `initial_tstep` is always written, because dry cells report it as their CFL step
  (`operators/dg2_update.cu:61`); a missing value makes dt collapse to 0.
* Time series are padded beyond `sim_time`, because the interpolation in
  `classes/PointSources.h:429-450` reads one row past the current one.
* A point inflow of Q m^3/s is written as Q/dx, because `mra/reinsert_point_srcs.cu:25`
  adds value*dt/dx to the free surface (the value is a unit-width discharge).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


# ----------------------------------------------------------------------------- writers

def _format_grid(values: np.ndarray, decimals: int) -> bytes:
    """Fast fixed-point ASCII formatting of a 2-D array, rows separated by newlines.

    Values are rounded to `decimals` places and printed as plain decimals; the
    result is byte-identical to '%.{decimals}f' for |v| < 1e12.
    """
    v = np.asarray(values, dtype=np.float64)
    scale = 10 ** decimals
    q = np.rint(v * scale).astype(np.int64)
    neg = q < 0
    a = np.abs(q)
    ip = a // scale
    fp = a % scale
    # integer part digits (up to 12), fraction digits fixed width
    nd_int = np.maximum(1, np.floor(np.log10(np.maximum(ip, 1))).astype(np.int64) + 1)
    width = nd_int + neg.astype(np.int64) + (1 + decimals if decimals > 0 else 0)
    rows, cols = v.shape
    # each value followed by a separator (space, or newline at row end)
    tot = width + 1
    offs = np.concatenate([[0], np.cumsum(tot.ravel())])
    out = np.full(int(offs[-1]), ord(" "), dtype=np.uint8)
    start = offs[:-1].reshape(rows, cols)
    flat_start = start.ravel()
    flat_neg = neg.ravel()
    flat_nd = nd_int.ravel()
    flat_ip = ip.ravel()
    flat_fp = fp.ravel()
    out[flat_start[flat_neg]] = ord("-")
    pos0 = flat_start + flat_neg.astype(np.int64)
    max_nd = int(flat_nd.max()) if flat_nd.size else 1
    for d in range(max_nd):
        has = flat_nd > d
        digit = (flat_ip // (10 ** (flat_nd - 1 - d).clip(0))) % 10
        out[(pos0 + d)[has]] = (ord("0") + digit[has]).astype(np.uint8)
    if decimals > 0:
        dot = pos0 + flat_nd
        out[dot] = ord(".")
        for d in range(decimals):
            digit = (flat_fp // 10 ** (decimals - 1 - d)) % 10
            out[dot + 1 + d] = (ord("0") + digit).astype(np.uint8)
    ends = (start + width)[:, -1]
    out[ends] = ord("\n")
    return out.tobytes()


def write_esri_ascii(path: str, grid_north_up: np.ndarray, cellsize: float,
                     xll: float = 0.0, yll: float = 0.0, decimals: int = 6) -> None:
    """Write an ESRI ASCII raster; `grid_north_up[0]` is the northernmost row."""
    nrows, ncols = grid_north_up.shape
    header = (f"ncols        {ncols}\nnrows        {nrows}\nxllcorner    {xll:g}\n"
              f"yllcorner    {yll:g}\ncellsize     {cellsize!r}\nNODATA_value -9999\n")
    with open(path, "wb") as fp:
        fp.write(header.encode())
        fp.write(_format_grid(grid_north_up, decimals))


@dataclass
class Case:
    """A generated case: the .par path plus what was generated (for tests and bench)."""
    par: str
    directory: str
    L: int
    solver: str
    cellsize: float
    sim_time: float
    dem: np.ndarray | None = None          # south-up (row 0 = south), shape (ysz, xsz)
    start_h: np.ndarray | None = None      # south-up
    meta: dict = field(default_factory=dict)


def _write_par(path: str, lines: list[str]) -> None:
    with open(path, "w") as fp:
        fp.write("\n".join(lines) + "\n")


def _common_par(solver: str, L: int, eps: float, sim_time: float, wall_height: float,
                manning: float, limitslopes: bool, tol_krivo: float, massint: float | None,
                saveint: float | None, cfl: float | None, extra: list[str]) -> list[str]:
    if solver not in ("mwdg2", "hwfv1"):
        raise ValueError("solver must be 'mwdg2' or 'hwfv1'")
    lines = [
        solver,
        "cuda",
        f"max_ref_lvl   {L}",
        f"epsilon       {eps!r}",
        f"wall_height   {wall_height!r}",
        "initial_tstep 1",
        f"fpfric        {manning!r}",
        f"sim_time      {sim_time!r}",
    ]
    if limitslopes:
        lines += ["limitslopes", f"tol_Krivo     {tol_krivo!r}"]
    if massint is not None:
        lines.append(f"massint       {massint!r}")
    if saveint is not None:
        lines.append(f"saveint       {saveint!r}")
    if cfl is not None:
        # Not read by the reference (its CFL is fixed in classes/SolverParams.cu:18,23).
        lines.append(f"CFL           {cfl!r}")
    return lines + extra


def _write_stage(path: str, points: list[tuple[float, float]]) -> None:
    with open(path, "w") as fp:
        fp.write(f"{len(points)}\n")
        for x, y in points:
            fp.write(f"{x!r} {y!r}\n")


# ----------------------------------------------------------------------------- cases

def circular_dam_break(directory: str, L: int = 8, solver: str = "mwdg2", eps: float = 1e-3,
                       sim_time: float = 3.5, domain: float = 50.0, radius: float = 2.5,
                       h_in: float = 2.5, h_out: float = 0.5, limitslopes: bool = True,
                       tol_krivo: float = 10.0, massint: float | None = 0.1,
                       cfl: float | None = None, manning: float = 0.0,
                       stage_points: list[tuple[float, float]] | None = None,
                       saveint: float | None = None, extra: list[str] | None = None) -> Case:
    """Circular dam break on a flat bed with closed walls (the 256^2 parity case's shape).

    The start raster holds h = h_in inside `radius` of the domain centre and h_out
    outside, sampled at raster-cell centres. The bed is 0 and `wall_height` is 100.
    `saveint` and `extra` (further .par lines, e.g. output keywords) pass through.
    """
    os.makedirs(directory, exist_ok=True)
    n = 1 << L
    dx = domain / n
    c = (np.arange(n) + 0.5) * dx
    X, Y = np.meshgrid(c, c)                       # Y increases northwards (south-up)
    r = np.hypot(X - domain / 2, Y - domain / 2)
    h = np.where(r < radius, h_in, h_out)
    dem = np.zeros((n, n))
    write_esri_ascii(os.path.join(directory, "case.dem"), dem[::-1], dx, decimals=1)
    write_esri_ascii(os.path.join(directory, "case.start"), h[::-1], dx, decimals=3)
    if stage_points is None:
        stage_points = [(domain / 2 + dx / 2, domain / 2 + dx / 2),
                        (domain / 2 + 5.0, domain / 2 + dx / 2),
                        (domain / 2 + 10.0, domain / 2 + 7.5),
                        (domain / 2 - 12.5, domain / 2 - 12.5)]
    _write_stage(os.path.join(directory, "case.stage"), stage_points)
    lines = _common_par(solver, L, eps, sim_time, 100.0, manning, limitslopes, tol_krivo,
                        massint, saveint, cfl,
                        ["DEMfile       case.dem", "startfile     case.start",
                         "stagefile     case.stage"] + list(extra or []))
    par = os.path.join(directory, "case.par")
    _write_par(par, lines)
    return Case(par=par, directory=directory, L=L, solver=solver, cellsize=dx,
                sim_time=sim_time, dem=dem, start_h=h,
                meta={"kind": "circular_dam_break", "radius": radius})


def fbm_surface(n: int, hurst: float, seed: int, relief: float) -> np.ndarray:
    """Fractional Brownian surface by spectral synthesis, rescaled to [0, relief].

    Amplitude ~ k^-(H+1) with uniformly random phases (PCG64 stream `seed`).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    kx = np.fft.fftfreq(n)[None, :]
    ky = np.fft.fftfreq(n)[:, None]
    k = np.hypot(kx, ky)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    phase = rng.uniform(0.0, 2.0 * np.pi, size=(n, n))
    spec = amp * np.exp(1j * phase)
    z = np.real(np.fft.ifft2(spec))
    z -= z.min()
    zmax = z.max()
    if zmax > 0:
        z *= relief / zmax
    return z


def fbm_catchment(directory: str, L: int = 12, solver: str = "mwdg2", eps: float = 1e-3,
                  sim_time: float = 7200.0, cellsize: float = 2.0, hurst: float = 0.8,
                  relief: float = 30.0, manning: float = 0.03, peak_q: float = 50.0,
                  t_peak: float = 1800.0, seed: int = 20261203, massint: float | None = None,
                  limitslopes: bool = False, tol_krivo: float = 10.0,
                  cfl: float | None = None, start_depth: np.ndarray | None = None,
                  stage_points: list[tuple[float, float]] | None = None,
                  saveint: float | None = None, extra: list[str] | None = None) -> Case:
    """fBm catchment with a west-edge point inflow (the 4096^2 benchmark case's shape).

    Dry start unless `start_depth` (south-up array) is given. The inflow is a
    triangular hydrograph 0 -> peak_q m^3/s at t_peak -> 0 at 2*t_peak, written as
    unit-width discharge peak_q/cellsize, padded to 2*sim_time + 2*t_peak.
    `saveint` and `extra` (further .par lines, e.g. output keywords) pass through.
    """
    os.makedirs(directory, exist_ok=True)
    n = 1 << L
    dem = fbm_surface(n, hurst, seed, relief)
    write_esri_ascii(os.path.join(directory, "case.dem"), dem[::-1], cellsize, decimals=3)
    user_extra = list(extra or [])
    extra = ["DEMfile       case.dem", "bcifile       case.bci", "bdyfile       case.bdy"]
    if start_depth is not None:
        write_esri_ascii(os.path.join(directory, "case.start"), start_depth[::-1], cellsize,
                         decimals=4)
        extra.append("startfile     case.start")
    y_src = (n // 2) * cellsize + cellsize / 2
    with open(os.path.join(directory, "case.bci"), "w") as fp:
        fp.write(f"P {cellsize / 2!r} {y_src!r} QVAR HYD\n")
    t_end = max(2.0 * sim_time, 2.0 * t_peak) + 2.0 * t_peak
    rows = [(0.0, 0.0), (peak_q / cellsize, t_peak), (0.0, 2.0 * t_peak), (0.0, t_end),
            (0.0, t_end + t_peak)]
    with open(os.path.join(directory, "case.bdy"), "w") as fp:
        fp.write("inflow hydrograph\nHYD\n")
        fp.write(f"{len(rows)} seconds\n")
        for v, t in rows:
            fp.write(f"{v!r} {t!r}\n")
    if stage_points is None:
        ext = n * cellsize
        stage_points = [(ext * 0.25 + cellsize / 2, ext * 0.5 + cellsize / 2),
                        (ext * 0.5 + cellsize / 2, ext * 0.5 + cellsize / 2)]
    _write_stage(os.path.join(directory, "case.stage"), stage_points)
    extra.append("stagefile     case.stage")
    lines = _common_par(solver, L, eps, sim_time, 1000.0, manning, limitslopes, tol_krivo,
                        massint, saveint, cfl, extra + user_extra)
    par = os.path.join(directory, "case.par")
    _write_par(par, lines)
    return Case(par=par, directory=directory, L=L, solver=solver, cellsize=cellsize,
                sim_time=sim_time, dem=dem, start_h=start_depth,
                meta={"kind": "fbm_catchment", "seed": seed, "hurst": hurst})


def lake_at_rest(directory: str, L: int = 7, solver: str = "mwdg2", eps: float = 1e-3,
                 sim_time: float = 1.0, cellsize: float = 1.0, level: float = 1.0,
                 relief: float = 0.8, seed: int = 7, manning: float = 0.0,
                 limitslopes: bool = False) -> Case:
    """Still water at surface `level` over an fBm bed (h = max(0, level - z))."""
    os.makedirs(directory, exist_ok=True)
    n = 1 << L
    dem = fbm_surface(n, 0.8, seed, relief)
    h = np.maximum(0.0, level - dem)
    write_esri_ascii(os.path.join(directory, "case.dem"), dem[::-1], cellsize, decimals=4)
    write_esri_ascii(os.path.join(directory, "case.start"), h[::-1], cellsize, decimals=4)
    lines = _common_par(solver, L, eps, sim_time, 1000.0, manning, limitslopes, 10.0,
                        None, None, None,
                        ["DEMfile       case.dem", "startfile     case.start"])
    par = os.path.join(directory, "case.par")
    _write_par(par, lines)
    return Case(par=par, directory=directory, L=L, solver=solver, cellsize=cellsize,
                sim_time=sim_time, dem=dem, start_h=h, meta={"kind": "lake_at_rest"})


def ensemble(root: str, n: int = 64, seed: int = 20261203, levels: tuple[int, ...] = (9, 10, 11),
             solver: str = "mwdg2", sim_time: float = 600.0, cellsize: float = 2.0) -> list[Case]:
    """Seeded ensemble of uneven scenarios, one folder each under `root`.

    Member i draws (PCG64 stream `seed`): max_ref_lvl uniformly from `levels`; an fBm DEM
    with Hurst ~ U(0.6, 0.9) over 0-30 m; with equal chance a dam break (depth 2.5 m inside
    a radius ~ U(0.05, 0.25) x domain around a random centre, 0.5 m outside, no inflow) or a
    dry start with a west-edge point inflow peaking at ~ U(5, 40) m^3/s at 300 s; Manning
    n ~ U(0.01, 0.05); epsilon 1e-3 or 1e-4.
    """
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L = int(rng.choice(levels))
        hurst = float(rng.uniform(0.6, 0.9))
        manning = float(rng.uniform(0.01, 0.05))
        eps = float(rng.choice([1e-3, 1e-4]))
        dam = bool(rng.integers(0, 2))
        m = 1 << L
        d = os.path.join(root, f"member{i:03d}")
        if dam:
            ext = m * cellsize
            radius = float(rng.uniform(0.05, 0.25)) * ext
            cx, cy = rng.uniform(0.25, 0.75, size=2) * ext
            c = (np.arange(m) + 0.5) * cellsize
            X, Y = np.meshgrid(c, c)
            depth = np.where(np.hypot(X - cx, Y - cy) < radius, 2.5, 0.5)
            case = fbm_catchment(d, L=L, solver=solver, eps=eps, sim_time=sim_time, cellsize=cellsize,
                                 hurst=hurst, manning=manning, peak_q=0.0, t_peak=300.0,
                                 seed=seed + i, start_depth=depth)
        else:
            peak = float(rng.uniform(5.0, 40.0))
            case = fbm_catchment(d, L=L, solver=solver, eps=eps, sim_time=sim_time, cellsize=cellsize,
                                 hurst=hurst, manning=manning, peak_q=peak, t_peak=300.0, seed=seed + i)
        case.meta.update({"member": i, "kind": "dam_break" if dam else "inflow", "eps": eps, "manning": manning})
        out.append(case)
    return out



def urban_surface(n: int, seed: int, hurst: float = 0.8, relief: float = 3.0, cover: float = 0.3,
                  block_height: tuple[float, float] = (5.0, 20.0), tile: int = 32,
                  block_side: tuple[int, int] = (8, 30)) -> np.ndarray:
    """fBm base (`relief` m) plus axis-aligned building blocks covering ~`cover` of the area.

    The domain is cut into `tile` x `tile` cell lots; a lot holds one block with the
    probability that makes the expected built fraction `cover`. A block's sides are drawn
    uniformly from `block_side` cells, its position uniformly inside the lot and its height
    uniformly from `block_height` m above the base (PCG64 stream `seed` + 1).
    """
    z = fbm_surface(n, hurst, seed, relief)
    t = min(tile, n)
    lo, hi = block_side
    hi = min(hi, t)
    lo = min(lo, hi)
    nt = n // t
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    w = rng.integers(lo, hi + 1, size=(nt, nt))
    d = rng.integers(lo, hi + 1, size=(nt, nt))
    x0 = (rng.random((nt, nt)) * (t - w + 1)).astype(np.int64)
    y0 = (rng.random((nt, nt)) * (t - d + 1)).astype(np.int64)
    mean_side = 0.5 * (lo + hi)
    p = min(1.0, cover * t * t / (mean_side * mean_side))
    on = rng.random((nt, nt)) < p
    height = rng.uniform(block_height[0], block_height[1], size=(nt, nt))
    li = np.arange(t)
    in_x = (li >= x0[..., None]) & (li < (x0 + w)[..., None])        # (lot row, lot col, cell col)
    in_y = (li >= y0[..., None]) & (li < (y0 + d)[..., None])        # (lot row, lot col, cell row)
    mask = in_y[:, :, :, None] & in_x[:, :, None, :] & on[:, :, None, None]
    add = np.where(mask, height[:, :, None, None], 0.0)              # (lot row, lot col, row, col)
    z[: nt * t, : nt * t] += add.transpose(0, 2, 1, 3).reshape(nt * t, nt * t)
    return z


def urban_catchment(directory: str, L: int = 13, solver: str = "mwdg2", eps: float = 1e-3,
                    sim_time: float = 3600.0, cellsize: float = 1.0, lake_level: float | None = 1.0,
                    peak_q: float = 100.0, t_rise: float = 900.0, manning: float = 0.03,
                    seed: int = 20261203, relief: float = 3.0, cover: float = 0.3,
                    limitslopes: bool = False, tol_krivo: float = 10.0, massint: float | None = None,
                    cfl: float | None = None) -> Case:
    """Urban catchment: `urban_surface` DEM, a lake at rest at `lake_level` (h =
    max(0, level - z) on the DEM as written, so h + z equals the level wherever water
    stands), and a west-edge point inflow rising linearly from 0 to `peak_q` m^3/s over
    `t_rise` seconds and held (unit-width value peak_q/cellsize). `lake_level` None is a
    dry start; `peak_q` 0 leaves the lake at rest.
    """
    os.makedirs(directory, exist_ok=True)
    n = 1 << L
    dem = np.round(urban_surface(n, seed, relief=relief, cover=cover), 3)
    write_esri_ascii(os.path.join(directory, "case.dem"), dem[::-1], cellsize, decimals=3)
    extra = ["DEMfile       case.dem", "bcifile       case.bci", "bdyfile       case.bdy"]
    start = None
    if lake_level is not None:
        start = np.maximum(0.0, np.round(lake_level - dem, 6))
        write_esri_ascii(os.path.join(directory, "case.start"), start[::-1], cellsize, decimals=6)
        extra.append("startfile     case.start")
    y_src = (n // 2) * cellsize + cellsize / 2
    with open(os.path.join(directory, "case.bci"), "w") as fp:
        fp.write(f"P {cellsize / 2!r} {y_src!r} QVAR HYD\n")
    t_end = 2.0 * max(sim_time, t_rise) + 2.0 * t_rise
    rows = [(0.0, 0.0), (peak_q / cellsize, t_rise), (peak_q / cellsize, t_end),
            (peak_q / cellsize, t_end + t_rise)]
    with open(os.path.join(directory, "case.bdy"), "w") as fp:
        fp.write("rising inflow\nHYD\n")
        fp.write(f"{len(rows)} seconds\n")
        for v, t in rows:
            fp.write(f"{v!r} {t!r}\n")
    ext = n * cellsize
    _write_stage(os.path.join(directory, "case.stage"),
                 [(ext * 0.25 + cellsize / 2, ext * 0.5 + cellsize / 2),
                  (ext * 0.5 + cellsize / 2, ext * 0.5 + cellsize / 2)])
    extra.append("stagefile     case.stage")
    lines = _common_par(solver, L, eps, sim_time, 1000.0, manning, limitslopes, tol_krivo,
                        massint, None, cfl, extra)
    par = os.path.join(directory, "case.par")
    _write_par(par, lines)
    return Case(par=par, directory=directory, L=L, solver=solver, cellsize=cellsize,
                sim_time=sim_time, dem=dem, start_h=start,
                meta={"kind": "urban_catchment", "seed": seed, "cover": cover})


def _write_series(path: str, series: dict[str, list[tuple[float, float]]]) -> None:
    """A .bdy file holding several named series (classes/Boundary.h:427-466): a comment
    line, then per series its name, "<rows> seconds" and "value time" rows."""
    with open(path, "w") as fp:
        fp.write("boundary series\n")
        for name, rows in series.items():
            fp.write(f"{name}\n{len(rows)} seconds\n")
            for v, t in rows:
                fp.write(f"{v!r} {t!r}\n")


# Boundary segments of each variant, one line per side (classes/Boundary.h:332-371 reads the
# first line starting with the side's letter; lower and upper are coordinates along the side).
BC_EDGE_VARIANTS = {
    "a": ["N 0 {ext} FREE", "E {q1} {q3} HFIX 1.3", "S {q1} {q3} QVAR SQ", "W 0 {ext} HVAR WH"],
    "b": ["N {q1} {q3} QFIX 0.4", "E 0 {ext} FREE", "S 0 {ext} HFIX 1.2", "W {q1} {q3} QVAR WQ"],
}


def bc_edges(directory: str, variant: str = "a", L: int = 7, solver: str = "mwdg2", eps: float = 1e-3,
             sim_time: float = 600.0, cellsize: float = 1.0, level: float = 1.0, relief: float = 0.8,
             seed: int = 11, manning: float = 0.02, limitslopes: bool = False) -> Case:
    """Still water at `level` over an fBm bed, driven through boundary segments.

    Variant "a": north FREE (whole side), east HFIX 1.3 m (middle half), south QVAR
    (middle half, series SQ rising to 0.6 m^2/s), west HVAR (whole side, series WH rising
    to 1.4 m). Variant "b": north QFIX 0.4 m^2/s (middle half), east FREE, south HFIX
    1.2 m, west QVAR (middle half, series WQ rising to 0.5 m^2/s). The series are padded
    far beyond `sim_time` (the reference reads one row past the current one).
    """
    os.makedirs(directory, exist_ok=True)
    n = 1 << L
    dem = fbm_surface(n, 0.8, seed, relief)
    h = np.maximum(0.0, level - dem)
    write_esri_ascii(os.path.join(directory, "case.dem"), dem[::-1], cellsize, decimals=4)
    write_esri_ascii(os.path.join(directory, "case.start"), h[::-1], cellsize, decimals=4)
    ext = n * cellsize
    fmt = {"ext": repr(ext), "q1": repr(ext / 4), "q3": repr(3 * ext / 4)}
    with open(os.path.join(directory, "case.bci"), "w") as fp:
        for line in BC_EDGE_VARIANTS[variant]:
            fp.write(line.format(**fmt) + "\n")
    pad = 4.0 * sim_time + 100.0
    _write_series(os.path.join(directory, "case.bdy"), {
        "WH": [(1.0, 0.0), (1.4, 2.0), (1.4, pad), (1.4, pad + 10.0)],
        "SQ": [(0.0, 0.0), (0.6, 2.0), (0.6, pad), (0.6, pad + 10.0)],
        "WQ": [(0.0, 0.0), (0.5, 1.5), (0.5, pad), (0.5, pad + 10.0)],
    })
    _write_stage(os.path.join(directory, "case.stage"), [(ext / 2 + cellsize / 2, ext / 2 + cellsize / 2)])
    lines = _common_par(solver, L, eps, sim_time, 1000.0, manning, limitslopes, 10.0, None, None, None,
                        ["DEMfile       case.dem", "startfile     case.start", "bcifile       case.bci",
                         "bdyfile       case.bdy", "stagefile     case.stage"])
    par = os.path.join(directory, "case.par")
    _write_par(par, lines)
    return Case(par=par, directory=directory, L=L, solver=solver, cellsize=cellsize, sim_time=sim_time,
                dem=dem, start_h=h, meta={"kind": "bc_edges", "variant": variant})


def start_q_nodata(directory: str, L: int = 7, solver: str = "mwdg2", eps: float = 1e-3,
                   sim_time: float = 600.0, cellsize: float = 1.0, xsz: int = 120, ysz: int = 100,
                   level: float = 1.0, relief: float = 0.8, seed: int = 13, wall_height: float = 5.0,
                   manning: float = 0.02, limitslopes: bool = True, nan_cell: bool = False) -> Case:
    """A lake over an fBm bed on an xsz x ysz DEM (narrower than the 2^L mesh) with a
    block of no-data (-9999) cells, which the reference reads as `wall_height`
    (input/read_raster_file.cpp:26-46), and a swirling initial discharge read from
    case.start.Qx / case.start.Qy (`startq2d`, input/read_and_project_modes_dg2.cu:42-49).
    The mesh outside the DEM keeps the bed at `wall_height` as well. `nan_cell` writes one
    depth of the start raster as "nan" (a corrupted input)."""
    os.makedirs(directory, exist_ok=True)
    n = 1 << L
    if xsz > n or ysz > n:
        raise ValueError("the DEM must fit the 2^L mesh")
    dem = fbm_surface(n, 0.8, seed, relief)[:ysz, :xsz]
    h = np.maximum(0.0, level - dem)
    yc, xc = (np.arange(ysz) + 0.5) * cellsize, (np.arange(xsz) + 0.5) * cellsize
    X, Y = np.meshgrid(xc, yc)
    qx = 0.2 * h * np.sin(2 * np.pi * Y / (ysz * cellsize))
    qy = -0.15 * h * np.sin(2 * np.pi * X / (xsz * cellsize))
    dem_out = np.round(dem, 4)
    block = (slice(ysz // 2 - 4, ysz // 2 + 4), slice(xsz // 3, xsz // 3 + 10))
    dem_out[block] = -9999.0
    h[block], qx[block], qy[block] = 0.0, 0.0, 0.0
    write_esri_ascii(os.path.join(directory, "case.dem"), dem_out[::-1], cellsize, decimals=4)
    write_esri_ascii(os.path.join(directory, "case.start"), h[::-1], cellsize, decimals=4)
    write_esri_ascii(os.path.join(directory, "case.start.Qx"), qx[::-1], cellsize, decimals=5)
    write_esri_ascii(os.path.join(directory, "case.start.Qy"), qy[::-1], cellsize, decimals=5)
    if nan_cell:
        path = os.path.join(directory, "case.start")
        lines = open(path).read().split("\n")
        row = lines[6 + ysz // 4].split(" ")
        row[xsz // 4] = "nan"
        lines[6 + ysz // 4] = " ".join(row)
        open(path, "w").write("\n".join(lines))
    _write_stage(os.path.join(directory, "case.stage"), [(xsz * cellsize / 4, ysz * cellsize / 4)])
    lines = _common_par(solver, L, eps, sim_time, wall_height, manning, limitslopes, 10.0, None, None, None,
                        ["DEMfile       case.dem", "startfile     case.start", "startq2d",
                         "stagefile     case.stage"])
    par = os.path.join(directory, "case.par")
    _write_par(par, lines)
    return Case(par=par, directory=directory, L=L, solver=solver, cellsize=cellsize, sim_time=sim_time,
                dem=dem_out, start_h=h, meta={"kind": "start_q_nodata", "xsz": xsz, "ysz": ysz})
