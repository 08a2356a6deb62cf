"""Keyword-deck writer for AM-CFD melt-pool runs.

Writes the reference's LS-DYNA-style input deck (keywords parsed by
src/sources/Mesh.cpp:39-435), the *MESH_FILE grid deck (Mesh.cpp:475-550) and,
for scanned paths, the 6-column toolpath file (t x y z on trackID;
DomainManager.cpp:268-289).  Every deck is synthetic: the shapes, sizes and
process parameters follow the benchmark configurations below, and the random
parameter sweep uses a fixed seed.

Conventions that the reference imposes on a deck:
- no blank lines (Mesh.cpp:50 reads line.at(0));
- acpa must be non-zero (CFDSolverManager.cpp:2562 divides by it); constant cp
  uses acpa = 1e-6 with hsmelt = acpa*Ts^2/2 + acpb*Ts and
  hlfriz = hlcal + L (DomainManager.cpp:251-254);
- the toolpath must extend past the final time (BoundCondManager.cpp:217-247
  leaves the beam position undefined otherwise).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

SEED = 20261203

Zone = Tuple[float, int, float]  # (length [m], control volumes, power exponent)


@dataclass
class Material:
    dens: float = 7800.0
    denl: float = 7800.0
    viscos: float = 6e-3
    tsolid: float = 1563.0
    tliquid: float = 1623.0
    latent: float = 2.7e5
    acpa: float = 1e-6
    acpb: float = 500.0
    acpl: float = 750.0
    thconsa: float = 0.0
    thconsb: float = 0.015
    thconsc: float = 15.0
    thconla: float = 0.015
    thconlb: float = 15.0

    def enthalpies(self) -> Tuple[float, float]:
        hsmelt = 0.5 * self.acpa * self.tsolid ** 2 + self.acpb * self.tsolid
        cpavg = (self.acpa * self.tsolid + self.acpb + self.acpl) * 0.5
        hlcal = hsmelt + cpavg * (self.tliquid - self.tsolid)
        return hsmelt, hlcal + self.latent


@dataclass
class Deck:
    name: str
    x_zones: Sequence[Zone]
    y_zones: Sequence[Zone]
    z_zones: Sequence[Zone]
    power: float = 200.0
    absorb: float = 0.35
    radius: float = 50e-6
    laser_factor: float = 2.0
    # single track: (lasertime, xstart, ystart, speed); toolpath: rows (t,x,y,z,on,id)
    single_track: Optional[Tuple[float, float, float, float]] = None
    toolpath: Optional[List[Tuple[float, float, float, float, int, int]]] = None
    material: Material = field(default_factory=Material)
    urf: Tuple[float, float, float, float, float] = (0.7, 0.7, 0.7, 0.7, 0.7)
    t_bound: Tuple[float, float, float, float, float] = (300.0, 300.0, 300.0, 300.0, 300.0)
    htc: Tuple[float, float, float, float, float] = (10.0, 10.0, 10.0, 10.0, 0.4)
    momentum: Tuple[float, float, float, float] = (5e-5, -4e-4, 1e8, -1.0)
    gravity: float = 9.8
    sigma: float = 5.67e-8
    t_amb: float = 300.0
    p_amb: float = 101.0e3
    gas_const: float = 8.314
    dt: float = 1e-5
    outtime: float = 1.0
    finaltime: float = 2e-3
    maxit: int = 20
    tol: float = 1e-5
    scheme: str = "power_law"  # power_law | exponential_law | upwind
    fluid_flow: bool = True
    # *BOUNDARY_EVAPORATION: (latent heat, evaporation T, factor, molar mass)
    evaporation: Optional[Tuple[float, float, float, float]] = None
    # *VOLUMETRIC_HEAT_SOURCE: (power, efficiency, thickness, radius, factor)
    volumetric: Optional[Tuple[float, float, float, float, float]] = None
    # *VOLUMETRIC_HEAT_SOURCE_TABLE rows (t, power, efficiency, thickness, radius, factor)
    heat_table: Optional[List[Tuple[float, float, float, float, float, float]]] = None
    # *CONTROL_TIMESTEP_VARIABLE rows (t, dt, output interval)
    vardt: Optional[List[Tuple[float, float, float]]] = None
    # *OUTPUT_FINAL_GEOMETRY file name (None: not requested)
    final_geometry: Optional[str] = None
    # *SOLVE_SPECIES: (initial concentration, mass diffusivity, partition coefficient kp,
    # under-relaxation urfc); its two fields are added to *SCALAR_OUT
    species: Optional[Tuple[float, float, float, float]] = None
    # *POWDER_BED_MODE: (layers, control volumes per layer, layer height, powder density,
    # powder cp a, cp b, powder conductivity a, b); csfrac and solfrac join *SCALAR_OUT
    powder: Optional[Tuple[int, int, float, float, float, float, float, float]] = None
    # *ACTIVATE_MOVING_MESH: 1-based numbers of the x and y zones that follow the beam
    moving_mesh: Optional[Tuple[int, int]] = None
    # *CALCULATE_SOLIDIFICATION_PARAMETERS: G and R (grad, rate) join *SCALAR_OUT
    solidification: bool = False
    # *TRACK_ENERGY_BASED_FREE_SURFACE: (lambda1, lambda2, surface tension, energy iterations,
    # energy tolerance, bisection iterations, bisection tolerance, under-relaxation); zr and
    # tempr join *SCALAR_OUT
    free_surface: Optional[Tuple[float, float, float, int, float, int, float, float]] = None

    @property
    def cells(self) -> Tuple[int, int, int]:
        return (sum(z[1] for z in self.x_zones), sum(z[1] for z in self.y_zones),
                sum(z[1] for z in self.z_zones))

    @property
    def steps(self) -> int:
        return int(math.ceil(self.finaltime / self.dt - 1e-9))

    def write(self, directory: str, relative: bool = False) -> str:
        """Write deck, mesh and toolpath files under `directory`; return the deck path.
        With relative=True the deck names its mesh/toolpath files without a
        directory (the reference opens them relative to the working directory)."""
        os.makedirs(directory, exist_ok=True)
        directory = os.path.abspath(directory)
        mesh = os.path.join(directory, f"{self.name}_mesh.k")
        ref = (lambda p: os.path.basename(p)) if relative else (lambda p: p)
        with open(mesh, "w") as f:
            for tag, zones in (("X", self.x_zones), ("Y", self.y_zones), ("Z", self.z_zones)):
                f.write(f"*{tag}_GRID_PARAMETERS\n$ zones / lengths / control volumes / exponents\n")
                f.write(f"  {len(zones)}\n")
                f.write("  " + " ".join(f"{z[0]:.10g}" for z in zones) + "\n")
                f.write("  " + " ".join(f"{int(z[1])}" for z in zones) + "\n")
                f.write("  " + " ".join(f"{z[2]:.10g}" for z in zones) + "\n")
        m = self.material
        hsmelt, hlfriz = m.enthalpies()
        lines = [
            "*KEYWORD_ID", self.name,
            "*DIRECTORY", ref(os.path.join(directory, "out")),
            "*PARAMETERS",
            f"accelGravity {self.gravity!r}", f"radBoltzmann {self.sigma!r}",
            f"ambientTemp {self.t_amb!r}", f"ambientPres {self.p_amb!r}",
            f"gasConstant {self.gas_const!r}",
            "*SCALAR_OUT", "temp", "uvel", "vvel", "wvel",
            *(["avgconcentration", "concentration"] if self.species is not None else []),
            *(["csfrac", "solfrac"] if self.powder is not None else []),
            *(["grad", "rate"] if self.solidification else []),
            *(["zr", "tempr"] if self.free_surface is not None else []),
            "*CONTROL_TERMINATION", "$ total_time max_iter nonlin_tolerance",
            f"  {self.finaltime!r} {self.maxit} {self.tol!r}",
            "*CONTROL_TIMESTEP", "$ sim_timestep output_timestep",
            f"  {self.dt!r} {self.outtime!r}",
            "*GAUSS_LASER_PARAMETERS", "$ power absorb radius factor",
            f"  {self.power!r} {self.absorb!r} {self.radius!r} {self.laser_factor!r}",
            "*MATERIAL_PROPERTIES", "$ dens denl viscos tsolid tliquid hsmelt hlfriz",
            f"  {m.dens!r} {m.denl!r} {m.viscos!r} {m.tsolid!r} {m.tliquid!r} {hsmelt!r} {hlfriz!r}",
            "$ acpa acpb acpl", f"  {m.acpa!r} {m.acpb!r} {m.acpl!r}",
            "$ thconsa thconsb thconsc thconla thconlb",
            f"  {m.thconsa!r} {m.thconsb!r} {m.thconsc!r} {m.thconla!r} {m.thconlb!r}",
            "*UNDER_RELAXATION", "$ urfu urfv urfw urfp urfh",
            "  " + " ".join(repr(float(v)) for v in self.urf),
            "*BOUNDARY_TEMPERATURES", "$ west east north bottom preheat",
            "  " + " ".join(repr(float(v)) for v in self.t_bound),
            "*BOUNDARY_ENERGY_EQUATION", "$ htci htcj htckl htckn emiss",
            "  " + " ".join(repr(float(v)) for v in self.htc),
            "*BOUNDARY_MOMENTUM_EQUATION", "$ beta dgdtp darcyKo a_oxygen",
            "  " + " ".join(repr(float(v)) for v in self.momentum),
        ]
        if self.scheme != "upwind":
            lines += ["*SELECT_DISCRETIZATION", self.scheme]
        if not self.fluid_flow:
            lines += ["*FLUID_FLOW_OFF"]
        if self.evaporation is not None:
            lines += ["*BOUNDARY_EVAPORATION", "  " + " ".join(repr(float(v)) for v in self.evaporation)]
        if self.volumetric is not None:
            lines += ["*VOLUMETRIC_HEAT_SOURCE", "  " + " ".join(repr(float(v)) for v in self.volumetric)]
        if self.species is not None:
            lines += ["*SOLVE_SPECIES", "$ initconc massdiff kp urfc",
                      "  " + " ".join(repr(float(v)) for v in self.species)]
        if self.moving_mesh is not None:
            lines += ["*ACTIVATE_MOVING_MESH", f"  {int(self.moving_mesh[0])} {int(self.moving_mesh[1])}"]
        if self.solidification:
            lines += ["*CALCULATE_SOLIDIFICATION_PARAMETERS"]
        if self.free_surface is not None:
            lines += ["*TRACK_ENERGY_BASED_FREE_SURFACE",
                      "$ lambda1 lambda2 surftens maxiter_energy tol_energy maxiter_bisect tol_bisect urf",
                      "  " + " ".join(repr(float(v)) for v in self.free_surface)]
        if self.powder is not None:
            nl, ncv, *rest = self.powder
            lines += ["*POWDER_BED_MODE", "$ numlayers ncvlayer layerheight density cpa cpb thcona thconb",
                      "  " + " ".join([str(int(nl)), str(int(ncv))] + [repr(float(v)) for v in rest])]
        if self.heat_table is not None:
            tab = os.path.join(directory, f"{self.name}_heat.txt")
            with open(tab, "w") as f:
                for row in self.heat_table:
                    f.write(" ".join(repr(float(v)) for v in row) + "\n")
            lines += ["*VOLUMETRIC_HEAT_SOURCE_TABLE", ref(tab)]
        if self.vardt is not None:
            tab = os.path.join(directory, f"{self.name}_dt.txt")
            with open(tab, "w") as f:
                for row in self.vardt:
                    f.write(" ".join(repr(float(v)) for v in row) + "\n")
            lines += ["*CONTROL_TIMESTEP_VARIABLE", ref(tab)]
        if self.final_geometry is not None:
            lines += ["*OUTPUT_FINAL_GEOMETRY", self.final_geometry]
        lines += ["*MESH_FILE", ref(mesh)]
        if self.toolpath is not None:
            crs = os.path.join(directory, f"{self.name}.crs")
            with open(crs, "w") as f:
                for t, x, y, z, on, tid in self.toolpath:
                    f.write(f"{t:.10e} {x:.10e} {y:.10e} {z:.10e} {int(on)} {int(tid)}\n")
            lines += ["*TOOLPATH_FILE", ref(crs)]
        else:
            st = self.single_track or (1.0, 0.5e-3, 1.0e-3, 1.0)
            lines += ["*SINGLE_TRACK_TOOL", "$ lasertime xstart ystart scanvel",
                      "  " + " ".join(repr(float(v)) for v in st)]
        path = os.path.join(directory, f"{self.name}.k")
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")
        return path


def _top(deck_z: Sequence[Zone]) -> float:
    return float(sum(z[0] for z in deck_z))


def powder_layers(name: str = "powder", nx: int = 16, ny: int = 10, nz: int = 8, tracks: int = 2,
                  track_steps: int = 4, dwell_steps: int = 2, power: float = 60.0, ncvzlayer: int = 2,
                  layerheight: float = 30e-6) -> Deck:
    """Powder-bed multi-layer deck on the small parity grid: one track per layer,
    alternating in x, the beam off for a dwell between layers.  The beam
    switching on activates the next layer (the first step included, the
    toolpath starting with the beam off), so numlayers = tracks + 1 keeps every
    activation inside the generated grid.  Powder: 90 % of the solid density,
    cp = 500 J/kg/K, k = 5 W/m/K.  On these 30 um cells the reference's outer
    iteration diverges (to NaN) for lighter or less conductive powder, or at
    100 W and above; this deck converges."""
    d = small(name, nx=nx, ny=ny, nz=nz, steps=1, power=power)
    lx, ly = 30e-6 * nx, 30e-6 * ny
    ztop = _top(d.z_zones)
    d.powder = (tracks + 1, ncvzlayer, layerheight, 0.9 * d.material.dens, 1e-6, 500.0, 0.0, 5.0)
    x0, x1, y = lx * 0.3, lx * 0.6, ly * 0.5
    rows = [(0.0, x0, y, ztop, 0, 1)]
    t, z, b = 0.0, ztop, x0
    for q in range(tracks):
        a, b = (x0, x1) if q % 2 == 0 else (x1, x0)
        z = ztop + (q + 1) * layerheight
        if q > 0:  # dwell with the beam off at the start of the next track
            t += dwell_steps * d.dt
            rows.append((t, a, y, z, 0, q + 1))
        t += track_steps * d.dt
        rows.append((t, b, y, z, 1, q + 1))
    rows.append((t + 10 * d.dt, b, y, z, 0, tracks))  # past the final time
    d.toolpath = rows
    d.single_track = None
    d.finaltime = t - 0.5 * d.dt
    return d


def moving_track(name: str = "moving", nx: int = 24, ny: int = 14, nz: int = 8, steps: int = 6,
                 power: float = 250.0, speed: float = 1.0, angle_deg: float = 30.0,
                 reverse: bool = False) -> Deck:
    """Moving-mesh deck on the small parity grid: three x zones (fine middle zone
    following the beam) over the small deck's three y zones, a straight toolpath
    at angle_deg to +x (towards -x and -y with reverse=True), G and R requested.
    A toolpath is needed: on the single-track path the reference never updates
    the beam's previous y position, so its y zones drift by ystart every step."""
    d = small(name, nx=nx, ny=ny, nz=nz, steps=steps, power=power)
    lx, ly = 30e-6 * nx, 30e-6 * ny
    nx1 = nx // 4
    d.x_zones = [(lx * 0.3, nx1, -1.2), (lx * 0.4, nx - 2 * nx1, 1.0), (lx * 0.3, nx1, 1.2)]
    d.moving_mesh = (2, 2)
    d.solidification = True
    ztop = _top(d.z_zones)
    a = math.radians(angle_deg + (180.0 if reverse else 0.0))
    x0, y0 = (lx * 0.35, ly * 0.4) if not reverse else (lx * 0.65, ly * 0.6)
    t_end = d.finaltime * 4
    d.toolpath = [(0.0, x0, y0, ztop, 0, 1),
                  (t_end, x0 + speed * t_end * math.cos(a), y0 + speed * t_end * math.sin(a), ztop, 1, 1)]
    d.single_track = None
    return d


def free_surface_track(name: str = "freesurf", steps: int = 4, power: float = 250.0) -> Deck:
    """The small parity deck with the energy-balance free surface: multiplier bracket
    [-1e5, 1e5], surface tension 1.8 N/m, 30 relaxation sweeps (tolerance 1e-6),
    up to 40 bisections to a volume residual of 1e-18 m^3, relaxation 0.5."""
    d = small(name, steps=steps, power=power)
    d.free_surface = (-1e5, 1e5, 1.8, 30, 1e-6, 40, 1e-18, 0.5)
    return d


def config0(steps: Optional[int] = None) -> Deck:
    """Plain FP64 single track along +x: 4.0 x 2.0 x 0.7 mm, 120 x 60 x 40 cells,
    refined toward the track (y = 1 mm) and the top surface; P = 200 W,
    r = 50 um, eta = 0.35, v = 1.0 m/s from (0.5, 1.0) mm; dt = 1e-5 s, 200 steps,
    <= 20 outer iterations, tolerance 1e-5."""
    d = Deck(name="config0",
             x_zones=[(4.0e-3, 120, 1.0)],
             y_zones=[(0.7e-3, 15, -1.5), (0.6e-3, 30, 1.0), (0.7e-3, 15, 1.5)],
             z_zones=[(0.5e-3, 15, -1.5), (0.2e-3, 25, 1.0)],
             single_track=(1.0, 0.5e-3, 1.0e-3, 1.0), finaltime=2e-3)
    if steps is not None:
        d.finaltime = (steps - 0.5) * d.dt
    return d


def diagonal_toolpath(x0, y0, ztop, speed, angle_deg, t_end):
    c, s = math.cos(math.radians(angle_deg)), math.sin(math.radians(angle_deg))
    return [(0.0, x0, y0, ztop, 0, 1),
            (t_end, x0 + speed * t_end * c, y0 + speed * t_end * s, ztop, 1, 1)]


def config1(steps: Optional[int] = None) -> Deck:
    """FP32-bulk / FP64-reduction case: 45-degree diagonal scan over a
    6.0 x 6.0 x 1.0 mm domain, 400 x 200 x 100 non-uniform cells (8 M);
    P = 300 W, r = 60 um, v = 0.8 m/s, dt = 5e-6 s, 500 steps."""
    zx = [(1.0e-3, 60, -1.2), (3.0e-3, 280, 1.0), (2.0e-3, 60, 1.2)]
    zy = [(1.0e-3, 30, -1.2), (3.0e-3, 140, 1.0), (2.0e-3, 30, 1.2)]
    zz = [(0.6e-3, 30, -1.5), (0.4e-3, 70, 1.0)]
    d = Deck(name="config1", x_zones=zx, y_zones=zy, z_zones=zz,
             power=300.0, radius=60e-6, dt=5e-6, finaltime=2.5e-3)
    d.toolpath = diagonal_toolpath(1.5e-3, 1.5e-3, _top(zz), 0.8, 45.0, 3.0e-3)
    if steps is not None:
        d.finaltime = (steps - 0.5) * d.dt
    return d


def config2(n: int = 64, seed: int = SEED, steps: int = 300) -> List[Deck]:
    """Process-parameter sweep: n single-track instances, grids drawn
    uniformly between 60 x 30 x 20 and 240 x 120 x 60 cells with the domain
    scaled from the config-0 domain by the same factor; P ~ U[100, 400] W,
    v ~ U[0.5, 1.5] m/s, r ~ U[40, 80] um; 300 steps each."""
    rng = np.random.default_rng(seed)
    decks = []
    for q in range(n):
        s = rng.uniform(0.0, 1.0)
        nx, ny, nz = int(round(60 + 180 * s)), int(round(30 + 90 * s)), int(round(20 + 40 * s))
        lx, ly, lz = 4.0e-3 * nx / 120, 2.0e-3 * ny / 60, 0.7e-3 * nz / 40
        P, v, rb = rng.uniform(100, 400), rng.uniform(0.5, 1.5), rng.uniform(40e-6, 80e-6)
        ny1 = ny // 4
        nz1 = int(round(nz * 0.375))
        d = Deck(name=f"sweep{q:02d}",
                 x_zones=[(lx, nx, 1.0)],
                 y_zones=[(ly * 0.35, ny1, -1.5), (ly * 0.30, ny - 2 * ny1, 1.0), (ly * 0.35, ny1, 1.5)],
                 z_zones=[(lz * 5 / 7, nz1, -1.5), (lz * 2 / 7, nz - nz1, 1.0)],
                 power=P, radius=rb, single_track=(1.0, lx * 0.125, ly * 0.5, v),
                 finaltime=(steps - 0.5) * 1e-5)
        decks.append(d)
    return decks


def config3_eval(steps: Optional[int] = None) -> Deck:
    """Held-out learned-warm-start evaluation: 200 x 100 x 60 single track,
    P = 250 W, v = 1.2 m/s, 1000 steps (domain scaled from config 0)."""
    lx, ly, lz = 4.0e-3 * 200 / 120, 2.0e-3 * 100 / 60, 0.7e-3 * 60 / 40
    d = Deck(name="config3", x_zones=[(lx, 200, 1.0)],
             y_zones=[(ly * 0.35, 25, -1.5), (ly * 0.3, 50, 1.0), (ly * 0.35, 25, 1.5)],
             z_zones=[(lz * 5 / 7, 22, -1.5), (lz * 2 / 7, 38, 1.0)],
             power=250.0, single_track=(1.0, lx * 0.1, ly * 0.5, 1.2), finaltime=1e-2)
    if steps is not None:
        d.finaltime = (steps - 0.5) * d.dt
    return d


def raster_toolpath(x0, x1, y0, hatch, tracks, ztop, speed, dwell, layers=2,
                    layer_dz=40e-6):
    """Bidirectional raster, `tracks` tracks per layer, laser off during the
    `dwell` between tracks; the second layer is rotated by 90 degrees (tracks
    along y) and raised by `layer_dz` in the beam z coordinate."""
    rows = [(0.0, x0, y0, ztop, 0, 1)]
    t = 0.0
    tid = 1
    for layer in range(layers):
        z = ztop + layer * layer_dz
        for tr in range(tracks):
            if layer % 2 == 0:
                y = y0 + tr * hatch
                a, b = (x0, x1) if tr % 2 == 0 else (x1, x0)
                p0, p1 = (a, y), (b, y)
            else:
                x = x0 + tr * hatch
                span = x1 - x0
                a, b = (y0, y0 + span) if tr % 2 == 0 else (y0 + span, y0)
                p0, p1 = (x, a), (x, b)
            # move (laser off) to the track start during the dwell
            t += dwell
            rows.append((t, p0[0], p0[1], z, 0, tid))
            t += abs(b - a) / speed
            rows.append((t, p1[0], p1[1], z, 1, tid))
            tid += 1
    rows.append((t + 1.0, rows[-1][1], rows[-1][2], rows[-1][3], 0, tid))
    return rows


def config4(steps: Optional[int] = None) -> Deck:
    """Multi-layer multi-track at scale: 10.0 x 5.0 x 1.2 mm, 600 x 300 x 120
    cells (21.6 M); 2 layers x 5 tracks, bidirectional raster, hatch 100 um,
    1 ms dwell, 90-degree rotation between layers; P = 200 W, v = 1.0 m/s,
    dt = 1e-5 s.  The second layer is a second pass over the same domain."""
    zx = [(3.0e-3, 100, -1.2), (4.0e-3, 400, 1.0), (3.0e-3, 100, 1.2)]
    zy = [(1.5e-3, 50, -1.2), (2.0e-3, 200, 1.0), (1.5e-3, 50, 1.2)]
    zz = [(0.8e-3, 40, -1.5), (0.4e-3, 80, 1.0)]
    d = Deck(name="config4", x_zones=zx, y_zones=zy, z_zones=zz, power=200.0)
    d.toolpath = raster_toolpath(3.2e-3, 6.8e-3, 2.3e-3, 100e-6, 5, _top(zz), 1.0, 1e-3)
    d.finaltime = d.toolpath[-2][0]
    if steps is not None:
        d.finaltime = (steps - 0.5) * d.dt
    return d


def small(name="small", nx=24, ny=14, nz=10, steps=6, power=300.0, speed=1.0,
          scheme="power_law", fluid_flow=True, toolpath=False, laser_off_after=None,
          maxit=20, urf=0.7) -> Deck:
    """A parity deck small enough for the single-threaded oracle to finish in
    about a second: 0.72 x 0.42 x 0.30 mm at the config-0 cell size near the
    track (30 um in x, 30 um in y, 20-30 um in z), power chosen to melt in the
    first step."""
    lx, ly = 30e-6 * nx, 30e-6 * ny
    nz2 = nz // 2 + 1
    zz = [(0.15e-3, nz - nz2, -1.2), (0.15e-3, nz2, 1.0)]
    ny1 = ny // 4
    zy = [(ly * 0.3, ny1, -1.2), (ly * 0.4, ny - 2 * ny1, 1.0), (ly * 0.3, ny1, 1.2)]
    d = Deck(name=name, x_zones=[(lx, nx, 1.0)], y_zones=zy, z_zones=zz, power=power,
             scheme=scheme, fluid_flow=fluid_flow, maxit=maxit, urf=(urf,) * 5)
    d.finaltime = (steps - 0.5) * d.dt
    lasertime = 1.0 if laser_off_after is None else laser_off_after * d.dt
    if toolpath:
        d.toolpath = diagonal_toolpath(lx * 0.3, ly * 0.35, _top(zz), speed, 30.0, d.finaltime * 4)
    else:
        d.single_track = (lasertime, lx * 0.3, ly * 0.5, speed)
    return d
