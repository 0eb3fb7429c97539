"""Seeded synthetic LS-EVPFFT inputs in the reference's file grammar.

Writes the four files the solver reads, in exactly the formats the reference's
own writers produce:

* microstructure ``.dat``: ``phi1 Phi phi2 i j k grain phase`` per voxel, Bunge
  angles in degrees (read by ``IO_functions.f90:759-761``);
* ``cuel.sx``: cubic 6x6 or isotropic ``E nu`` (``utils/io_utils.py:36-70``);
* ``cupl2.sx``: FCC {111}<110> slip with Voce parameters
  (``utils/io_utils.py:73-122``);
* ``fft.in``: the deck grammar of ``utils/sim_cases/creep_calibration.py`` and
  ``utils/sim_cases/tension.py`` (parsed by ``IO_functions.f90:6-365``).

Microstructures are periodic Voronoi tessellations (minimum-image distance)
from ``numpy.random.default_rng(seed)`` seeds, with orientations uniform on
SO(3): phi1, phi2 ~ U[0, 360), Phi = arccos(U[-1, 1]).  These stand in for the
reference's shipped ``micro1.dat`` (no other microstructures are shipped).
"""
from __future__ import annotations

import dataclasses
import math
from pathlib import Path

import numpy as np

FCC_SLIP = [
    (1, 1, -1, 0, 1, 1),
    (1, 1, -1, 1, 0, 1),
    (1, 1, -1, 1, -1, 0),
    (1, -1, -1, 0, 1, -1),
    (1, -1, -1, 1, 0, 1),
    (1, -1, -1, 1, 1, 0),
    (1, -1, 1, 0, 1, 1),
    (1, -1, 1, 1, 0, -1),
    (1, -1, 1, 1, 1, 0),
    (1, 1, 1, 0, 1, -1),
    (1, 1, 1, 1, 0, -1),
    (1, 1, 1, 1, -1, 0),
]


# BCC {110}<111> and {112}<111>: 24 systems in two modes (plane normal, slip direction)
BCC_110 = [(0, 1, 1, 1, 1, -1), (0, 1, 1, 1, -1, 1), (0, 1, -1, 1, 1, 1), (0, 1, -1, -1, 1, 1),
           (1, 0, 1, 1, 1, -1), (1, 0, 1, -1, 1, 1), (1, 0, -1, 1, 1, 1), (1, 0, -1, 1, -1, 1),
           (1, 1, 0, 1, -1, 1), (1, 1, 0, -1, 1, 1), (1, -1, 0, 1, 1, 1), (1, -1, 0, 1, 1, -1)]
BCC_112 = [(1, 1, 2, 1, 1, -1), (-1, 1, 2, 1, -1, 1), (1, -1, 2, -1, 1, 1), (1, 1, -2, 1, 1, 1),
           (1, 2, 1, 1, -1, 1), (-1, 2, 1, 1, 1, -1), (1, 2, -1, -1, 1, 1), (1, -2, 1, 1, 1, 1),
           (2, 1, 1, -1, 1, 1), (-2, 1, 1, 1, 1, 1), (2, 1, -1, 1, -1, 1), (2, -1, 1, 1, 1, -1)]


@dataclasses.dataclass
class Material:
    c11: float = 250000.0
    c12: float = 150000.0
    c44: float = 120000.0
    nrs: float = 10.0
    gamd0: float = 1e-3
    tau0f: float = 100.0
    tau0b: float = 100.0
    tau1: float = 40.0
    thet0: float = 500.0
    thet1: float = 20.0
    hself: float = 1.0
    hlat: float = 1.4
    slip: str = "fcc"  # "fcc": {111}<110>, 12 systems; "bcc24": {110}<111> + {112}<111>, 24 systems in two modes


@dataclasses.dataclass
class Loading:
    """One process block of fft.in."""

    kind: str = "creep"  # "creep" (sigma33 controlled) or "tension" (udot33 controlled)
    stress33: float = 150.0
    udot33: float = 1e-3  # tension: imposed rate; creep: initial-guess rate (the template writes 1e-4)
    tdot: float = 10.0
    tdotmin: float | None = None  # default: equal to tdot (fixed increment count)
    nsteps: int = 100
    error: float = 1e-5
    erroral: float = 1e-9
    itmax: int = 200
    iupdate: int = 1
    iuphard: int = 1
    iwfields: int = 0
    iwstep: int = 0
    xc0: float = 2.0
    igamma: int = 0
    ictrl: int = -1
    thermo_file: str | None = None  # ITHERMO = 1 with this per-grain eigenstrain file


def _nearest_seed(pts: np.ndarray, seeds: np.ndarray, box: np.ndarray) -> np.ndarray:
    """1-based index of the nearest seed under the minimum-image (periodic) distance; exact
    ties go to the lowest seed index."""
    try:
        from scipy.spatial import cKDTree
    except ImportError:  # pragma: no cover - scipy is part of the environment
        cKDTree = None
    if cKDTree is not None and len(seeds) > 1:
        tree = cKDTree(np.mod(seeds, box), boxsize=box)
        dist, idx = tree.query(pts, k=2)
        tie = dist[:, 0] == dist[:, 1]
        best = np.where(tie, np.minimum(idx[:, 0], idx[:, 1]), idx[:, 0])
        return best.astype(np.int64) + 1
    best = np.full(pts.shape[0], np.inf)
    grain = np.zeros(pts.shape[0], dtype=np.int64)
    for g in range(len(seeds)):
        d = pts - seeds[g]
        d -= box * np.round(d / box)
        r2 = np.einsum("ij,ij->i", d, d)
        m = r2 < best
        best[m] = r2[m]
        grain[m] = g + 1
    return grain


def voronoi_micro(n: int | tuple[int, int, int], ngrains: int, seed: int, phase2_spheres: float = 0.0,
                  sphere_r: tuple[float, float] = (2.0, 4.0)):
    """Return (grain[n1,n2,n3], phase[...], euler[ngrains,3] in degrees).

    Grain ids are 1-based; the voxel index order is (i, j, k) = (x, y, z)."""
    n1, n2, n3 = (n, n, n) if isinstance(n, int) else n
    rng = np.random.default_rng(seed)
    seeds = rng.uniform(0.0, 1.0, size=(ngrains, 3)) * np.array([n1, n2, n3])
    phi1 = rng.uniform(0.0, 360.0, ngrains)
    Phi = np.degrees(np.arccos(rng.uniform(-1.0, 1.0, ngrains)))
    phi2 = rng.uniform(0.0, 360.0, ngrains)
    euler = np.stack([phi1, Phi, phi2], axis=1)
    ii, jj, kk = np.meshgrid(np.arange(n1) + 0.5, np.arange(n2) + 0.5, np.arange(n3) + 0.5, indexing="ij")
    pts = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)
    box = np.array([n1, n2, n3], dtype=float)
    grain = _nearest_seed(pts, seeds, box).reshape(n1, n2, n3)
    phase = np.ones((n1, n2, n3), dtype=np.int64)
    if phase2_spheres > 0.0:
        target = phase2_spheres * n1 * n2 * n3
        count = 0
        while count < target:
            c = rng.uniform(0.0, 1.0, 3) * box
            r = rng.uniform(*sphere_r)
            # voxel centres within the sphere's bounding box, wrapped periodically (same test as over the whole grid)
            lo = np.floor(c - r - 0.5).astype(int)
            hi = np.ceil(c + r - 0.5).astype(int)
            ax = [np.arange(lo[a], hi[a] + 1) for a in range(3)]
            gi, gj, gk = np.meshgrid(*ax, indexing="ij")
            d = np.stack([gi + 0.5 - c[0], gj + 0.5 - c[1], gk + 0.5 - c[2]], axis=-1)
            d -= box * np.round(d / box)
            inside = np.einsum("...i,...i->...", d, d) <= r * r
            wi, wj, wk = gi[inside] % n1, gj[inside] % n2, gk[inside] % n3
            fresh = phase[wi, wj, wk] != 2
            count += np.unique((wi[fresh] * n2 + wj[fresh]) * n3 + wk[fresh]).size  # voxels newly in phase 2
            phase[wi, wj, wk] = 2
    return grain, phase, euler


def write_micro(path: Path, grain, phase, euler, euler2=None) -> None:
    """Write ``phi1 Phi phi2 i j k grain phase`` lines, x index fastest."""
    n1, n2, n3 = grain.shape
    lines = []
    for k in range(n3):
        for j in range(n2):
            for i in range(n1):
                g = int(grain[i, j, k])
                p = int(phase[i, j, k])
                e = euler[g - 1] if (p == 1 or euler2 is None) else euler2
                lines.append(f"{e[0]:.6f} {e[1]:.6f} {e[2]:.6f} {i + 1} {j + 1} {k + 1} {g} {p}")
    Path(path).write_text("\n".join(lines) + "\n")


def write_cuel(path: Path, m: Material | None = None, iso: int = 0, young: float = 400000.0, nu: float = 0.3) -> None:
    if iso == 0:
        m = m or Material()
        txt = (f"0 \t\t\t\t\tISO\n"
               f"{m.c11} {m.c12} {m.c12} 0.0 0.0 0.0\n"
               f"{m.c12} {m.c11} {m.c12} 0.0 0.0 0.0\n"
               f"{m.c12} {m.c12} {m.c11} 0.0 0.0 0.0\n"
               f"0.0 0.0 0.0 {m.c44} 0.0 0.0\n"
               f"0.0 0.0 0.0 0.0 {m.c44} 0.0\n"
               f"0.0 0.0 0.0 0.0 0.0 {m.c44}\n")
    else:
        txt = f"1 \t\t\t\t\tISO\n{young}   {nu}   YOUNG(MPa),NU (V+R/2)\n"
    Path(path).write_text(txt)


def write_cupl2(path: Path, m: Material) -> None:
    if m.slip == "bcc24":
        _write_cupl2_bcc(path, m)
        return
    rows = "\n".join(f"{a}    {b}   {c}      {d}    {e}    {f}" for a, b, c, d, e, f in FCC_SLIP)
    txt = ("SLIP SYSTEMS FOR CUBIC CRYSTAL\n"
           "CUBIC          icryst\n"
           "1.   1.   1.   crystal axes (cdim(i))\n"
           "1              nmodesx (total # of modes listed in the file)\n"
           "1              nmodes  (# of modes to be used in the calculation)\n"
           "1              mode(i) (label of the modes to be used)\n"
           "{111}<110>   SLIP\n"
           f"1   12   {m.nrs:.8f}   {m.gamd0:.8e}   0.0  0                 modex,nsmx,nrsx,gamd0x,twshx,isectwx\n"
           f"{m.tau0f!r}  {m.tau0b!r}   {m.tau1!r}   {m.thet0!r}  {m.thet1!r}  0  tau0xf,tau0xb,tau1x,thet0,thet1,hpfac\n"
           f"{m.hself!r}   {m.hlat!r}                                               hselfx,hlatex\n"
           f"{rows}\n")
    Path(path).write_text(txt)


def _write_cupl2_bcc(path: Path, m: Material) -> None:
    """Two modes with the same power law and Voce parameters; latent hardening hlat between and within modes."""
    txt = ("SLIP SYSTEMS FOR CUBIC CRYSTAL (BCC)\n"
           "CUBIC          icryst\n"
           "1.   1.   1.   crystal axes (cdim(i))\n"
           "2              nmodesx (total # of modes listed in the file)\n"
           "2              nmodes  (# of modes to be used in the calculation)\n"
           "1  2           mode(i) (label of the modes to be used)\n")
    for mode, (name, rows) in enumerate((("{110}<111>", BCC_110), ("{112}<111>", BCC_112)), start=1):
        txt += (f"{name}   SLIP\n"
                f"{mode}   12   {m.nrs:.8f}   {m.gamd0:.8e}   0.0  0                 modex,nsmx,nrsx,gamd0x,twshx,isectwx\n"
                f"{m.tau0f!r}  {m.tau0b!r}   {m.tau1!r}   {m.thet0!r}  {m.thet1!r}  0  tau0xf,tau0xb,tau1x,thet0,thet1,hpfac\n"
                f"{m.hself!r}   {m.hlat!r}   {m.hlat!r}                                 hselfx,hlatex(1:2)\n")
        txt += "\n".join(f"{a}    {b}   {c}      {d}    {e}    {f}" for a, b, c, d, e, f in rows) + "\n"
    Path(path).write_text(txt)


def _process_block(p: Loading) -> str:
    if p.kind == "creep":
        iudot = "\t0       1       1           iudot     |    flag for vel.grad. \n" \
                "\t1       0       1                     |    (0:unknown-1:known)        \n" \
                "\t1       1       0                     |            \n"
        udot33 = p.udot33
        iscau = "\t1       0        0           iscau    |    flag for Cauchy            \n" \
                "\t\t\t1        0                    |                               \n" \
                "\t\t\t\t\t 1                    |                               \n"
        s33 = p.stress33
    elif p.kind == "tension":
        iudot = "\t0       1       1           iudot     |    flag for vel.grad. \n" \
                "\t1       0       1                     |    (0:unknown-1:known)        \n" \
                "\t1       1       1                     |            \n"
        udot33 = p.udot33
        iscau = "\t1       0        0           iscau    |    flag for Cauchy            \n" \
                "\t\t\t1        0                    |                               \n" \
                "\t\t\t\t\t 0                    |                               \n"
        s33 = 0.0
    else:
        raise ValueError(p.kind)
    tmin = p.tdot if p.tdotmin is None else p.tdotmin
    return ("*INFORMATION ABOUT TEST CONDITIONS                                                            \n"
            "* boundary conditions                                                     \n"
            + iudot +
            "\t\t\t\t\t\t\t\t\t\t  |                               \n"
            f"\t0.0     0.0      0.0          udot    |    vel.grad                   \n"
            f"\t0.0     0.0      0.0                  |                               \n"
            f"\t0.0     0.0      {udot33!r}               |                                      \n"
            "\t\t\t\t\t\t\t\t\t\t  |                               \n"
            + iscau +
            "\t\t\t\t\t\t\t\t\t\t  |                               \n"
            "\t0.      0.       0.          scauchy  |    Cauchy stress              \n"
            "\t\t\t0.       0.                   |                               \n"
            f"\t\t\t\t\t {s33!r}                  @                               \n"
            "* other                                                                   \n"
            f"{p.tdot!r} {p.tdot!r} {tmin!r} 0.5  eqincr or tdot, tdotref, tdotmin, devmmx\n"
            f"{p.ictrl}                     ictrl (1-6: strain comp, 0: VM eq, -1: tdot)\n"
            "*INFORMATION ABOUT RUN CONDITIONS                                         \n"
            f"{p.nsteps}               nsteps (total number of time steps)     \n"
            f"{p.error!r} {p.erroral!r}  err,erral (tolerances for fields and Augm.Lagr.)\n"
            f"{p.itmax}             itmax (maximum allowed number of iterations)\n"
            "0               IRECOVER read grain states from STRESS.IN  (1) or not (0)?      \n"
            "0               ISAVE write grain states in STRESS.OUT (1) or not (0)?                    \n"
            f"{p.iupdate}               IUPDATE update tex & RVE dim (1) or not (0)?\n"
            f"{p.iuphard}               IUPHARD\n"
            "1               IWTEX (write texture at the end)\n"
            f"{p.iwfields} {p.iwstep}            IWFIELDS,IWSTEP (write fields, and frequency of writing)\n"
            f"{p.xc0!r} {p.igamma}            XC0, IGAMMA (0-continious,1-discrete central diff,2-rotated)\n"
            + ("0               ITHERMO (if ithermo=1, next line is filethermo)\n" if p.thermo_file is None else
               f"1               ITHERMO (if ithermo=1, next line is filethermo)\n{p.thermo_file}\n"))


def write_fft_in(path: Path, n, micro: Path, cupl2: Path, cuel: Path, processes: list[Loading],
                 phase2: tuple[int, Path, Path] | None = None, complgas: float = 0.0,
                 dispini: tuple[int, Path] | None = None) -> None:
    n1, n2, n3 = (n, n, n) if isinstance(n, int) else n
    nph = 1 if phase2 is None else 2
    txt = (f"{nph}                      number of phases (nph)\n"
           f"{n1} {n2} {n3}               nx,ny,nz - number of points\n"
           "1.  1.  1.             RVE dimensions (delt) - keep as 1.0 1.0 1.0\n"
           "* name and path of microstructure file (filetext)\n"
           f"{micro}\n"
           "*INFORMATION ABOUT PHASE #1\n"
           "0                          igas(iph)\n"
           "* name and path of single crystal files (dummy if igas(iph)=1)\n"
           f"{cupl2}\n{cuel}\n")
    if phase2 is not None:
        igas, pl2, el2 = phase2
        txt += ("*INFORMATION ABOUT PHASE #2\n"
                f"{igas}                          igas(iph)\n"
                "* name and path of single crystal files (dummy if igas(iph)=1)\n"
                f"{pl2}\n{el2}\n")
    txt += ("* restart analysis, remeshing and gas phase compliance\n"
            "0 200                  ires,imicrosave\n"
            f"{complgas}                   complgas (% of stiffness)\n"
            "* initial displacement field\n"
            + ("0                      IDISPINI (if idispini=1, next line is filedispl)\n" if dispini is None else
               f"{dispini[0]}                      IDISPINI (if idispini=1, next line is filedispl)\n{dispini[1]}\n") +
            f"{len(processes)}                      number of processes (nproc)\n")
    for p in processes:
        txt += _process_block(p)
    Path(path).write_text(txt)


@dataclasses.dataclass
class Case:
    name: str
    n: int
    ngrains: int
    seed: int
    material: Material
    processes: list
    phase2_frac: float = 0.0
    phase2_gas: bool = False  # the second phase as gas (igas = 1) instead of the stiff elastic phase
    complgas: float = 0.0
    thermo_eigenstrain: float = 0.0  # > 0: per-grain thermal eigenstrain of this size (ITHERMO = 1)
    dispini: int = 0  # 1: initial displacement at cell centres, 2: at nodes (IDISPINI)
    dispini_amp: float = 0.05  # amplitude of that displacement field, in voxels


def case_c1(nsteps: int = 100) -> Case:
    """16^3 creep, 64 grains, n=10, sigma33=150 MPa, dt=10 s, tol 1e-5."""
    return Case("creep16", 16, 64, 1, Material(nrs=10.0),
                [Loading(kind="creep", stress33=150.0, udot33=1e-4, tdot=10.0, nsteps=nsteps, error=1e-5, erroral=1e-9, itmax=200)])


def case_c2(nsteps: int = 200, n: int = 64, ngrains: int = 500) -> Case:
    """64^3 tension, 500 grains, n=20, udot33=1e-3/s, dt=0.5 s (10 % strain in 200 increments)."""
    return Case(f"tension{n}", n, ngrains, 2, Material(nrs=20.0),
                [Loading(kind="tension", udot33=1e-3, tdot=0.5, nsteps=nsteps, error=1e-5, erroral=1e-9, itmax=200)])


def case_c3(stress33: float = 150.0, nsteps: int = 300, n: int = 128, ngrains: int = 2000) -> Case:
    """128^3 creep, 2000 grains + 5 vol% stiff isotropic phase 2 (E=400 GPa, nu=0.3, tau0=1e8: elastic only)."""
    return Case(f"creep{n}_2ph", n, ngrains, 3, Material(nrs=10.0),
                [Loading(kind="creep", stress33=stress33, udot33=1e-4, tdot=10.0, nsteps=nsteps, error=1e-5, erroral=1e-9, itmax=200)],
                phase2_frac=0.05)


def write_case(case: Case, root: Path, micro_cache: dict | None = None) -> Path:
    """Write every input file of ``case`` under ``root``; returns the fft.in path."""
    root = Path(root)
    root.mkdir(parents=True, exist_ok=True)
    grain, phase, euler = voronoi_micro(case.n, case.ngrains, case.seed, phase2_spheres=case.phase2_frac)
    micro = root / "micro.dat"
    write_micro(micro, grain, phase, euler, euler2=(0.0, 0.0, 0.0))
    write_cuel(root / "cuel.sx", case.material)
    write_cupl2(root / "cupl2.sx", case.material)
    phase2 = None
    if case.phase2_frac > 0.0:
        write_cuel(root / "cuel2.sx", iso=1, young=400000.0, nu=0.3)
        m2 = dataclasses.replace(case.material, tau0f=1e8, tau0b=1e8)
        write_cupl2(root / "cupl2_2.sx", m2)
        phase2 = (1 if case.phase2_gas else 0, root / "cupl2_2.sx", root / "cuel2.sx")
    processes = case.processes
    if case.thermo_eigenstrain > 0.0:
        write_thermo(root / "thermo.txt", case.ngrains, case.thermo_eigenstrain, case.seed)
        processes = [dataclasses.replace(p, thermo_file=str(root / "thermo.txt")) for p in processes]
    dispini = None
    if case.dispini:
        write_dispini(root / "disp.txt", case.n, case.dispini, case.dispini_amp, case.seed)
        dispini = (case.dispini, root / "disp.txt")
    fft = root / "fft.in"
    write_fft_in(fft, case.n, micro, root / "cupl2.sx", root / "cuel.sx", processes, phase2=phase2,
                 complgas=case.complgas, dispini=dispini)
    return fft


def write_dispini(path: Path, n, kind: int, amp: float, seed: int) -> None:
    """Initial displacement file read after IDISPINI (IO_functions.f90:850-880): one line
    ``i j k u1 u2 u3`` per cell centre (kind 1, i fastest) or per node (kind 2, (n+1) per axis,
    one z plane when n3 = 1).  The field is a smooth periodic one: a sum of three seeded
    sine modes of amplitude ``amp`` voxels per component."""
    n1, n2, n3 = (n, n, n) if isinstance(n, int) else n
    rng = np.random.default_rng([seed, 11])
    kvec = rng.integers(1, 3, size=(3, 3, 3))  # component, mode, axis
    phase = rng.uniform(0.0, 2.0 * np.pi, size=(3, 3))
    off = 0.5 if kind == 1 else 0.0  # cell centres sit half a voxel from the nodes
    m1, m2 = (n1, n2) if kind == 1 else (n1 + 1, n2 + 1)
    m3 = n3 if kind == 1 else (1 if n3 == 1 else n3 + 1)
    k, j, i = np.meshgrid(np.arange(m3), np.arange(m2), np.arange(m1), indexing="ij")
    x = (i + off) / n1, (j + off) / n2, (k + off) / n3
    u = np.zeros((3,) + i.shape)
    for c in range(3):
        for mo in range(3):
            arg = 2 * np.pi * sum(kvec[c, mo, a] * x[a] for a in range(3)) + phase[c, mo]
            u[c] += amp / 3.0 * np.sin(arg)
    lines = [f"{a + 1} {b + 1} {cc + 1} {u0:.15e} {u1:.15e} {u2:.15e}"
             for cc, b, a, u0, u1, u2 in zip(k.ravel(), j.ravel(), i.ravel(), u[0].ravel(), u[1].ravel(), u[2].ravel())]
    Path(path).write_text("\n".join(lines) + "\n")


def write_thermo(path: Path, ngrains: int, size: float, seed: int) -> None:
    """Per-grain thermal eigenstrain file read after ITHERMO = 1: the grain count, then one line
    of e11 e22 e33 e23 e13 e12 per grain (seeded, components uniform in [-size, size])."""
    rng = np.random.default_rng([seed, 7])
    e = rng.uniform(-size, size, size=(ngrains, 6))
    lines = [str(ngrains)] + [" ".join(f"{x:.10e}" for x in row) for row in e]
    Path(path).write_text("\n".join(lines) + "\n")


def case_c4(i: int, nsteps: int = 150) -> Case:
    """Solve i of the batched calibration sweep (seed 1000 + i): grid edge from {16, 32, 48, 64},
    32-500 grains, tau0 log-uniform in [50, 200] MPa, n uniform in [5, 20], theta0 log-uniform in
    [100, 1000] MPa (theta1 = 20 <= theta0, as the reference requires); creep at 120 MPa."""
    rng = np.random.default_rng(1000 + i)
    n = int(rng.choice([16, 32, 48, 64]))
    ngr = int(rng.integers(32, 501))
    tau0 = float(math.exp(rng.uniform(math.log(50.0), math.log(200.0))))
    nrs = float(rng.uniform(5.0, 20.0))
    thet0 = float(math.exp(rng.uniform(math.log(100.0), math.log(1000.0))))
    mat = Material(nrs=nrs, tau0f=tau0, tau0b=tau0, thet0=thet0)
    return Case(f"sweep{i}", n, ngr, 1000 + i, mat,
                [Loading(kind="creep", stress33=120.0, udot33=1e-4, tdot=10.0, nsteps=nsteps, error=1e-5, erroral=1e-9,
                         itmax=200)])


ARRHENIUS_Q = 250e3  # J/mol
GAS_R = 8.314462618  # J/(mol K)


def case_c5(i: int, increments_scale: float = 1.0) -> Case:
    """Request i of the served stream (seed stream 5): grid edge exp(U[ln 16, ln 96]) rounded to a
    multiple of 8; temperature from {475, 525, 575} (taken as kelvin: the reference has no
    temperature model) scaling gamma0 = 1e-3 exp(-Q/R (1/T - 1/525)) with Q = 250 kJ/mol; creep
    stress U[80, 220] MPa; U{50..400} increments (times increments_scale, at least 1); 32-500 grains,
    at most one per 8 voxels."""
    rng = np.random.default_rng([5, i])
    edge = int(round(math.exp(rng.uniform(math.log(16.0), math.log(96.0))) / 8.0) * 8)
    edge = min(max(edge, 16), 96)
    temp = float(rng.choice([475.0, 525.0, 575.0]))
    gamd0 = 1e-3 * math.exp(-ARRHENIUS_Q / GAS_R * (1.0 / temp - 1.0 / 525.0))
    stress = float(rng.uniform(80.0, 220.0))
    nsteps = max(1, int(round(int(rng.integers(50, 401)) * increments_scale)))
    ngr = min(int(rng.integers(32, 501)), edge ** 3 // 8)
    mat = Material(nrs=10.0, gamd0=gamd0)
    return Case(f"stream{i}_T{int(temp)}", edge, ngr, 5000 + i, mat,
                [Loading(kind="creep", stress33=stress, udot33=1e-4, tdot=10.0, nsteps=nsteps, error=1e-5, erroral=1e-9,
                         itmax=200)])


def stream_arrivals(k: int, rate_per_s: float = 20.0, seed: int = 5) -> np.ndarray:
    """Arrival times (s) of the first k requests of a Poisson stream."""
    rng = np.random.default_rng([seed, 99])
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=k))
