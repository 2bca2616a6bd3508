"""Seeded synthetic systems written in the reference's input formats.

A system is a directory with the files the reference reads: ``control``
(RDCONTROL.f90), ``interaction`` plus one two-column table file per entry
(RDINTERACT.f90), ``coordinate`` (RDCOOR.f90) and, for hybrid systems,
``virtual`` (RDVIRTUAL.f90), ``virtbonds`` (RDVIRTBONDS.f90) and
``virtangles`` (RDVIRTANGLES.f90).  Units are the files' units: nm, ps,
kJ/mol, degrees, kg/mol.

``lj_fluid``, ``polymer_melt`` and ``cg_melt`` build the benchmark
workloads (single-type LJ fluid, bead-spring melt, large CG melt); ``feature_mix``
builds a small system that exercises every term the step supports
(bonds, angles, torsions, out-of-planes, exclusions with non_bonded 4 and 5,
explicit beads, centre and centre-of-mass virtual sites, virtbonds,
virtangles, MTS, NPT).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

KB_KJ = 0.0083144626  # kJ/mol/K


@dataclass
class Tab:
    fname: str
    x: np.ndarray
    v: np.ndarray


@dataclass
class SystemSpec:
    control: dict
    types: list                      # [(name, mass kg/mol, 'A'|'B')]
    pos: np.ndarray                  # (N,3) nm, unwrapped
    vel: np.ndarray                  # (N,3) nm/ps
    itype: np.ndarray                # (N,) 1-based
    bonds: list                      # adjacency lists, 1-based partners, <=4 each
    molecules: list                  # [(name, count)] in particle order
    box: tuple
    bond_tabs: list = field(default_factory=list)     # [((a,b), Tab)]
    angle_tabs: list = field(default_factory=list)    # [((a,b,c), Tab)]
    torsion_tabs: list = field(default_factory=list)  # [((a,b,c,d), Tab)]
    nb_tabs: list = field(default_factory=list)       # [((a,b), Tab)]
    oop_tabs: list = field(default_factory=list)      # [((a,b,c,d), Tab)]
    virtual: list = field(default_factory=list)       # [(vtype, [members 1-based], centre or 0)]
    virtbonds: list = field(default_factory=list)     # [(i, j)] global 1-based
    virtangles: list = field(default_factory=list)    # [(i, j, k, t)]


CONTROL_ORDER = [
    "ensemble", "temperature", "pressure", "atoms", "num_of_time_steps", "time_step",
    "temperature_coupling_time", "pressure_coupling_time", "isothermal_compressibility",
    "virtual_sites", "mts", "bead_cutoff", "bead_neighbour_list_cutoff", "non_bonded_bead",
    "cutoff", "neighbour_list_cutoff", "update_neighbour_list", "trajectory", "halt_drift",
    "non_bonded", "initialize_velocities",
]


def _fmt(x) -> str:
    return repr(float(np.float32(x)))


def write_system(spec: SystemSpec, directory: str) -> str:
    os.makedirs(directory, exist_ok=True)
    c = dict(spec.control)
    with open(os.path.join(directory, "control"), "w") as f:
        for k in CONTROL_ORDER:
            if k in c:
                f.write(f"{k:<27}{c[k]}\n")
        f.write("end\n")
    written = set()

    def table(t: Tab):
        if t.fname in written:
            return
        written.add(t.fname)
        with open(os.path.join(directory, t.fname), "w") as f:
            for a, b in zip(t.x, t.v):
                f.write(f"{a:.9e}  {b:.9e}\n")

    with open(os.path.join(directory, "interaction"), "w") as f:
        f.write(f"atom_types {len(spec.types)}\n# type label mass A/B\n")
        for i, (name, mass, lab) in enumerate(spec.types, 1):
            f.write(f"  {i}  {name}  {mass:.8g}  {lab}\n")
        for key, tabs in (("bond_types", spec.bond_tabs), ("angle_types", spec.angle_tabs),
                          ("torsion_types", spec.torsion_tabs),
                          ("non_bonded_interaction_types", spec.nb_tabs), ("Out_of_Planes", spec.oop_tabs)):
            f.write(f"{key} {len(tabs)}\n# types file\n")
            for types, t in tabs:
                table(t)
                f.write("  " + "  ".join(str(x) for x in types) + f"  {t.fname}\n")
    n = spec.pos.shape[0]
    lines = [" " + "*" * 70,
             " ********** Time    0.0000000000000000       (ps)",
             " ********** Box Length(X, Y, Z in nanometres)                **********",
             "   " + "   ".join(_fmt(b) for b in spec.box),
             " " + "*" * 70,
             " ********** Record for each atom is in the form:-            **********",
             " ********** Index Atom_Type No._of_bonds X Y Z (coords.in nm) *******",
             " ********** Vx Vy Vz (in nm/ps) Indices_of_bonded_atoms         *******",
             " " + "*" * 70,
             f" num_of_molecules: {len(spec.molecules)}"]
    # REAL*4 values to 9 significant digits, which read back to the same REAL*4
    pos = spec.pos.astype(np.float32).astype(np.float64).tolist()
    vel = spec.vel.astype(np.float32).astype(np.float64).tolist()
    itype = [int(t) for t in spec.itype]
    labels = [t[2] for t in spec.types]
    i = 0
    out = []
    for m, (name, cnt) in enumerate(spec.molecules, 1):
        out.append(f" {cnt} atoms_in_molecule_no. {m} {name}")
        for _ in range(cnt):
            b = spec.bonds[i]
            p, v, t = pos[i], vel[i], itype[i]
            out.append(" %d %d %d %.9g %.9g %.9g %s" % (i + 1, t, len(b), p[0], p[1], p[2], labels[t - 1]))
            out.append("   %.9g %.9g %.9g  " % (v[0], v[1], v[2]) + " ".join(map(str, b)))
            i += 1
    assert i == n
    with open(os.path.join(directory, "coordinate"), "w") as f:
        f.write("\n".join(lines + out) + "\n")
    if spec.virtual:
        with open(os.path.join(directory, "virtual"), "w") as f:
            f.write(" **********synthetic\n # Number of virtual sites:\n")
            f.write(f" {len(spec.virtual)}\n Type of VS, Natoms in VS, Centre or 0 for COM\n Members\n")
            for k, (vt, mem, ctr) in enumerate(spec.virtual, 1):
                f.write(f" {k} {vt} {len(mem)} {ctr}\n " + " ".join(str(x) for x in mem) + "\n")
    if spec.virtbonds:
        with open(os.path.join(directory, "virtbonds"), "w") as f:
            for a, b in spec.virtbonds:
                f.write(f"{a} {b}\n")
    if spec.virtangles:
        with open(os.path.join(directory, "virtangles"), "w") as f:
            for a, b, cc, t in spec.virtangles:
                f.write(f"{a} {b} {cc} {t}\n")
    return directory


# ------------------------------------------------------------------ tables
def lj_table(fname, sigma, eps, rmax, dr, vcap=1.0e20):
    n = int(round(rmax / dr)) + 1
    r = np.arange(n) * dr
    with np.errstate(divide="ignore", over="ignore"):
        sr6 = (sigma / np.where(r > 0, r, 1.0)) ** 6
        v = 4.0 * eps * (sr6 * sr6 - sr6)
    v[0] = v[1]
    v = np.minimum(v, vcap)
    return Tab(fname, r, v)


def shifted_force_lj_table(fname, sigma, eps, rc, dr):
    """LJ 12-6 with its value and slope shifted to zero at the cutoff rc, so
    that the energy is continuous and conserved to the integrator's order."""
    t = lj_table(fname, sigma, eps, rc, dr)
    sr6 = (sigma / rc) ** 6
    vc = 4.0 * eps * (sr6 * sr6 - sr6)
    dvc = 4.0 * eps * (-12.0 * sr6 * sr6 + 6.0 * sr6) / rc
    v = t.v - vc - (t.x - rc) * dvc
    v[0] = v[1]
    return Tab(fname, t.x, v)


def perturbed_lj_table(fname, sigma, eps, rmax, dr, amps):
    t = lj_table(fname, sigma, eps, rmax, dr)
    r = t.x
    add = sum(a * np.sin((k + 1) * np.pi * r / rmax) for k, a in enumerate(amps))
    return Tab(fname, r, t.v + add)


def harmonic_bond_table(fname, r0, k, rmax, dr):
    n = int(round(rmax / dr)) + 1
    r = np.arange(n) * dr
    return Tab(fname, r, 0.5 * k * (r - r0) ** 2)


def harmonic_angle_table(fname, theta0_deg, k, dtheta=0.18):
    n = int(round(180.0 / dtheta)) + 1
    th = np.arange(n) * dtheta
    return Tab(fname, th, 0.5 * k * np.radians(th - theta0_deg) ** 2)


def cosine_torsion_table(fname, k, mult=3, dphi=1.8):
    n = int(round(360.0 / dphi)) + 1
    ph = np.arange(n) * dphi
    return Tab(fname, ph, k * (1.0 + np.cos(np.radians(mult * ph))))


def oop_table(fname, k, dphi=1.8):
    # signed out-of-plane angle, tabulated from -180 (first row, index 0 after the
    # row-0 rule keeps it) to 180 degrees
    n = int(round(360.0 / dphi)) + 1
    ph = -180.0 + np.arange(n) * dphi
    return Tab(fname, ph, 0.5 * k * np.radians(ph) ** 2)


def maxwell_boltzmann(rng, masses_kg_mol, temp):
    sd = np.sqrt(KB_KJ * temp / (np.asarray(masses_kg_mol) * 1000.0))  # nm/ps
    v = rng.normal(size=(len(masses_kg_mol), 3)) * sd[:, None]
    m = np.asarray(masses_kg_mol)[:, None]
    v -= (m * v).sum(0) / m.sum()
    return v


# ----------------------------------------------------------- placements
def random_fluid(rng, n, box, dmin):
    """Uniform positions in [-L/2, L/2)^3 with rejection below dmin (cell grid)."""
    L = float(box)
    nc = max(1, int(L / dmin))
    cs = L / nc
    grid: dict = {}
    pts = np.zeros((n, 3))
    k = 0
    tries = 0
    while k < n:
        p = (rng.random(3) - 0.5) * L
        c = tuple(((p + L / 2) / cs).astype(int) % nc)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get(((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc), ()):
                        d = p - pts[q]
                        d -= L * np.round(d / L)
                        if d @ d < dmin * dmin:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
        tries += 1
        if ok or tries > 200 * n:
            grid.setdefault(c, []).append(k)
            pts[k] = p
            k += 1
    return pts


def random_walk_chains(rng, nchains, nper, box, bond, theta_deg, dmin, max_tries=100, max_restarts=50):
    """Chains grown bead by bead with fixed bond length and bond angle and a
    random dihedral.  A bead may not come closer than dmin to any earlier bead
    except its two bonded predecessors; a chain that cannot continue is
    restarted from a new random point."""
    L = float(box)
    nc = max(1, int(L / max(dmin, 1e-3)))
    cs = L / nc
    grid: dict = {}
    n = nchains * nper
    pts = np.zeros((n, 3))
    th = math.radians(theta_deg)

    def cell(p):
        return tuple((((p + L / 2) % L) / cs).astype(int) % nc)

    def clear(p, k, first):
        c = cell(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get(((c[0] + dx) % nc, (c[1] + dy) % nc, (c[2] + dz) % nc), ()):
                        if q >= k - 2 and q >= first:
                            continue
                        d = p - pts[q]
                        d -= L * np.round(d / L)
                        if d @ d < dmin * dmin:
                            return False
        return True

    k = 0
    for ch in range(nchains):
        start = k
        for restart in range(max_restarts + 1):
            k = start
            placed = []
            ok_chain = True
            for b in range(nper):
                ok = False
                for t in range(max_tries):
                    if b == 0:
                        p = (rng.random(3) - 0.5) * L
                    elif b == 1:
                        u = rng.normal(size=3)
                        p = pts[k - 1] + bond * u / np.linalg.norm(u)
                    else:
                        a, bb = pts[k - 2], pts[k - 1]
                        u = bb - a
                        u /= np.linalg.norm(u)
                        w = rng.normal(size=3)
                        w -= (w @ u) * u
                        w /= np.linalg.norm(w)
                        p = bb + bond * (math.cos(math.pi - th) * u + math.sin(math.pi - th) * w)
                    if clear(p, k, start):
                        ok = True
                        break
                if not ok and restart < max_restarts:
                    ok_chain = False
                    break
                pts[k] = p
                c = cell(p)
                grid.setdefault(c, []).append(k)
                placed.append((c, k))
                k += 1
            if ok_chain:
                break
            for c, q in placed:  # undo the partial chain
                grid[c].remove(q)
    return pts


def chain_bonds(nchains, nper, offset=0):
    bonds = []
    for ch in range(nchains):
        base = offset + ch * nper
        for b in range(nper):
            nb = []
            if b > 0:
                nb.append(base + b)  # previous (1-based id of base+b-1 is base+b)
            if b < nper - 1:
                nb.append(base + b + 2)
            bonds.append(nb)
    return bonds


def _all_angle_keys(types):
    keys = []
    for b in types:
        for a in types:
            for c in types:
                if a <= c:
                    keys.append((a, b, c))
    return keys


def _all_torsion_keys(types):
    keys, seen = [], set()
    for a in types:
        for b in types:
            for c in types:
                for d in types:
                    k, r = (a, b, c, d), (d, c, b, a)
                    if r in seen or k in seen:
                        continue
                    seen.add(k)
                    keys.append(k)
    return keys


# ------------------------------------------------------------------ configs
def lj_fluid(n=4000, rho=8.0, seed=1, nsteps=1000, dmin=0.3, shifted=False, dt=0.010):
    """Single-type LJ bead fluid: uniform positions rejected below dmin, LJ
    sigma 0.47 nm.  (With dmin 0.3 nm the first steps at dt 10 fs meet pair
    forces beyond the fixed-point range; a larger dmin avoids that.)"""
    rng = np.random.default_rng(seed)
    box = (n / rho) ** (1.0 / 3.0)
    pos = random_fluid(rng, n, box, dmin)
    mass = 0.072
    vel = maxwell_boltzmann(rng, [mass] * n, 300.0)
    control = dict(ensemble="NVE", temperature=300, pressure=101.3, atoms=n, num_of_time_steps=nsteps,
                   time_step=dt, temperature_coupling_time="0.1D0", pressure_coupling_time="5.0D0",
                   isothermal_compressibility="1.0D-6", virtual_sites=0, mts=0, bead_cutoff=1.2,
                   bead_neighbour_list_cutoff=1.4, non_bonded_bead=4, cutoff=1.2, neighbour_list_cutoff=1.4,
                   update_neighbour_list=10, trajectory=nsteps, halt_drift=nsteps + 1, non_bonded=4,
                   initialize_velocities="N")
    return SystemSpec(control=control, types=[("CG", mass, "A")], pos=pos, vel=vel, itype=np.ones(n, int),
                      bonds=[[] for _ in range(n)], molecules=[("bead", 1)] * n, box=(box, box, box),
                      nb_tabs=[((1, 1), (shifted_force_lj_table if shifted else lj_table)("nb11", 0.47, 3.5, 1.2,
                                                                                          0.002))])


def polymer_melt(nchains=400, nper=100, rho=20.0, ntypes=3, seed=2, nsteps=5000, temp=500.0, dt=0.001,
                 rcut=1.0, rlist=1.2, nupdate=10, ensemble="NVT", mass=0.014, bond=0.153, theta0=112.0):
    """Bead-spring melt with tabulated bond/angle/torsion: 400 chains x 100 beads by default."""
    rng = np.random.default_rng(seed)
    n = nchains * nper
    box = (n / rho) ** (1.0 / 3.0)
    pos = random_walk_chains(rng, nchains, nper, box, bond, theta0, 0.8 * 0.30)
    itype = np.array([1 + (k % ntypes) for ch in range(nchains) for k in range(nper)])
    vel = maxwell_boltzmann(rng, [mass] * n, temp)
    types = list(range(1, ntypes + 1))
    sig = {t: 0.30 + 0.10 * (t - 1) / max(1, ntypes - 1) for t in types}
    bond_t = harmonic_bond_table("bond.tab", bond, 2.5e5, 0.3, 0.0003)
    ang_t = harmonic_angle_table("ang.tab", theta0, 500.0)
    tor_t = cosine_torsion_table("tors.tab", 5.0)
    control = dict(ensemble=ensemble, temperature=temp, pressure=101.3, atoms=n, num_of_time_steps=nsteps,
                   time_step=dt, temperature_coupling_time="0.1D0", pressure_coupling_time="5.0D0",
                   isothermal_compressibility="1.0D-6", virtual_sites=0, mts=0, bead_cutoff=rcut,
                   bead_neighbour_list_cutoff=rlist, non_bonded_bead=4, cutoff=rcut, neighbour_list_cutoff=rlist,
                   update_neighbour_list=nupdate, trajectory=nsteps, halt_drift=nsteps + 1, non_bonded=4,
                   initialize_velocities="N")
    return SystemSpec(
        control=control, types=[(f"C{t}", mass, "A") for t in types], pos=pos, vel=vel, itype=itype,
        bonds=chain_bonds(nchains, nper), molecules=[("chain", nper)] * nchains, box=(box, box, box),
        bond_tabs=[((a, b), bond_t) for a in types for b in types if a <= b],
        angle_tabs=[(k, ang_t) for k in _all_angle_keys(types)],
        torsion_tabs=[(k, tor_t) for k in _all_torsion_keys(types)],
        nb_tabs=[((a, b), lj_table(f"nb{a}{b}", 0.5 * (sig[a] + sig[b]), 0.5, rcut, 0.002))
                 for a in types for b in types if a <= b])


def cg_melt(nchains=10000, nper=200, rho=8.0, seed=4, nsteps=2000, ntypes=4):
    """Large CG melt for the roofline study: 10,000 chains x 200 beads (2,000,000)
    by default, 4 bead types by position along the chain, at number density rho.
    The chains follow a serpentine path through a cubic lattice of spacing
    rho^(-1/3) (bonds at their rest length, no overlaps), so the set-up is
    vectorised and fast at any size.  Harmonic bond (rest length = spacing) and
    angle (150 deg, weak) tables; the 10 type-pair LJ tables are tabulated on a
    0.001 nm grid to the 1.4 nm cutoff (list 1.6 nm, rebuilt every 10 steps);
    NVT 300 K, dt 10 fs."""
    rng = np.random.default_rng(seed)
    n = nchains * nper
    a = rho ** (-1.0 / 3.0)
    m = int(np.ceil(n ** (1.0 / 3.0)))
    box = m * a
    pos = serpentine_lattice(m)[:n] * a - 0.5 * box + 0.5 * a
    # alternate z offsets bend the chains along x
    pos[:, 2] += 0.1 * a * (np.arange(n) % 2 - 0.5)
    pos += rng.normal(scale=0.01, size=pos.shape)
    types = list(range(1, ntypes + 1))
    itype = np.tile(1 + np.arange(nper) % ntypes, nchains)
    mass = 0.072
    vel = maxwell_boltzmann(rng, np.full(n, mass), 300.0)
    control = dict(ensemble="NVT", temperature=300.0, pressure=101.3, atoms=n, num_of_time_steps=nsteps,
                   time_step=0.010, temperature_coupling_time="0.1D0", pressure_coupling_time="5.0D0",
                   isothermal_compressibility="1.0D-6", virtual_sites=0, mts=0, bead_cutoff=1.4,
                   bead_neighbour_list_cutoff=1.6, non_bonded_bead=4, cutoff=1.4, neighbour_list_cutoff=1.6,
                   update_neighbour_list=10, trajectory=nsteps, halt_drift=nsteps + 1, non_bonded=4,
                   initialize_velocities="N")
    bond_t = harmonic_bond_table("bond.tab", a, 5.0e3, 1.0, 0.001)
    ang_t = harmonic_angle_table("ang.tab", 150.0, 10.0)
    return SystemSpec(
        control=control, types=[(f"C{t}", mass, "A") for t in types], pos=pos, vel=vel, itype=itype,
        bonds=chain_bonds(nchains, nper), molecules=[("chain", nper)] * nchains, box=(box, box, box),
        bond_tabs=[((i, j), bond_t) for i in types for j in types if i <= j],
        angle_tabs=[(k, ang_t) for k in _all_angle_keys(types)],
        nb_tabs=[((i, j), lj_table(f"nb{i}{j}", 0.42 + 0.01 * (i + j), 2.0, 1.4, 0.001)) for i in types for j in types
                 if i <= j])


def feature_mix(seed=7, nmol=6, ensemble="NVT", nmts=0, non_bonded=4, temp=400.0):
    """A small hybrid system exercising every supported term.

    Each molecule is a backbone of atoms (label A) with a three-bonded branch
    point per monomer (out-of-plane terms) and two coarse-grained beads
    (label B) bonded to its ends; every monomer carries one virtual site, on a
    centre atom or at its centre of mass.  virtbonds exclude each bead from
    its own molecule's sites and one virtangle couples a bead to two sites.
    Molecules lie on separate lattice rows, so no two particles overlap.
    """
    rng = np.random.default_rng(seed)
    types = [("C", 0.012, "A"), ("H", 0.001008, "A"), ("N", 0.014, "A"), ("B1", 0.043, "B"),
             ("B2", 0.040, "B"), ("V1", 0.05, "B"), ("V2", 0.05, "B")]
    mono = [1, 3, 2, 1]  # C N H C; N carries H and the second C
    nmono = 4
    box = 3.2
    pos, itype, bonds, mols, virt, vb, va = [], [], [], [], [], [], []
    slots = rng.permutation(25)[:nmol]
    for m in range(nmol):
        start = len(itype)
        iy, iz = divmod(int(slots[m]), 5)
        y0, z0 = -1.4 + 0.6 * iy, -1.4 + 0.6 * iz
        x0 = -1.0 + 0.4 * rng.random()
        for k in range(nmono):
            for t in mono:
                itype.append(t)
                bonds.append([])
        for k in range(nmono):
            c1, n1, h1, c2 = [start + 4 * k + j + 1 for j in range(4)]
            for a, b in ((c1, n1), (n1, h1), (n1, c2)):
                bonds[a - 1].append(b)
                bonds[b - 1].append(a)
            if k + 1 < nmono:
                nxt = start + 4 * (k + 1) + 1
                bonds[c2 - 1].append(nxt)
                bonds[nxt - 1].append(c2)
        # planar zig-zag backbone c1-n1-c2-c1'... (bond 0.11 nm, angle 115 deg);
        # H on N along the bisector, beads continuing the zig-zag at both ends
        nat = 4 * nmono
        dx, dy = 0.11 * math.sin(math.radians(57.5)), 0.5 * 0.11 * math.cos(math.radians(57.5))
        xyz = [None] * (nat + 2)
        for k in range(nmono):
            for q, slot in enumerate((0, 1, 3)):  # c1, n1, c2 are backbone sites 3k, 3k+1, 3k+2
                bidx = 3 * k + q
                sgn = 1.0 if bidx % 2 == 0 else -1.0
                xyz[4 * k + slot] = np.array([x0 + dx * bidx, y0 + sgn * dy, z0])
            n_ = xyz[4 * k + 1]
            sgn = 1.0 if (3 * k + 1) % 2 == 0 else -1.0
            xyz[4 * k + 2] = n_ + np.array([0.0, sgn * 0.11, 0.0])
        xyz[nat] = np.array([x0 - dx, y0 - dy, z0])
        last = 3 * nmono - 1
        xyz[nat + 1] = np.array([x0 + dx * (last + 1), y0 + (dy if (last + 1) % 2 == 0 else -dy), z0])
        for p_ in xyz:
            pos.append(p_ + rng.normal(scale=0.008, size=3))
        b1, b2 = len(itype) + 1, len(itype) + 2
        itype += [4, 5]
        bonds += [[], []]
        for a, b in ((start + 1, b1), (start + 4 * (nmono - 1) + 4, b2)):
            bonds[a - 1].append(b)
            bonds[b - 1].append(a)
        mols.append((f"mol{m + 1}", nat + 2))
        for k in range(nmono):
            members = [start + 4 * k + j + 1 for j in range(4)]
            virt.append((6, members, members[1]) if k % 2 == 0 else (7, members, 0))
    natoms = len(itype)
    for m in range(nmol):
        first = sum(c for _, c in mols[:m])
        beads = (first + 4 * nmono + 1, first + 4 * nmono + 2)
        sites = [natoms + m * nmono + k + 1 for k in range(nmono)]
        for bd in beads:
            for v in sites:
                vb.append((bd, v))
        va.append((beads[0], sites[0], sites[1], 1))
    pos = np.array(pos)
    masses = [types[t - 1][1] for t in itype]
    vel = maxwell_boltzmann(rng, masses, temp)
    at, bt = [1, 2, 3], [4, 5, 6, 7]
    all_t = at + bt
    bond_t = harmonic_bond_table("bond.tab", 0.11, 1.5e5, 0.6, 0.0003)
    ang_t = harmonic_angle_table("ang.tab", 115.0, 300.0)
    tor_t = cosine_torsion_table("tors.tab", 4.0)
    oop_t = oop_table("oop.tab", 40.0)
    bond_keys = sorted({tuple(sorted((itype[i], itype[j - 1]))) for i in range(natoms) for j in bonds[i]})
    control = dict(ensemble=ensemble, temperature=temp, pressure=101.3, atoms=natoms, num_of_time_steps=100,
                   time_step=0.0005, temperature_coupling_time="0.1D0", pressure_coupling_time="1.0D0",
                   isothermal_compressibility="4.5D-5", virtual_sites=len(virt), mts=nmts, bead_cutoff=0.9,
                   bead_neighbour_list_cutoff=1.0, non_bonded_bead=non_bonded, cutoff=0.7,
                   neighbour_list_cutoff=0.8, update_neighbour_list=5, trajectory=100, halt_drift=7,
                   non_bonded=non_bonded, initialize_velocities="N")
    nb_tabs = []
    for a in all_t:
        for b in all_t:
            if a <= b:
                both_cg = a in bt and b in bt
                rc = 0.9 if both_cg else 0.7
                sig = 0.35 if both_cg else 0.25
                nb_tabs.append(((a, b), perturbed_lj_table(f"nb{a}_{b}", sig, 0.8, rc + 0.1, 0.002,
                                                           [0.1, -0.05, 0.02])))
    return SystemSpec(
        control=control, types=types, pos=pos, vel=vel, itype=np.array(itype), bonds=bonds, molecules=mols,
        box=(box, box, box), bond_tabs=[(k, bond_t) for k in bond_keys],
        angle_tabs=[(k, ang_t) for k in _all_angle_keys(all_t)],
        torsion_tabs=[(k, tor_t) for k in _all_torsion_keys(at)],
        nb_tabs=nb_tabs,
        oop_tabs=[((3, 1, 2, 1), oop_t), ((3, 1, 1, 2), oop_t)],
        virtual=virt, virtbonds=vb, virtangles=va)


def hybrid_melt(n_atomistic=100, n_cg=100, nmono=20, seed=3, nsteps=10000, nmts=9, temp=300.0):
    """Hybrid atomistic/CG melt with centre-of-mass virtual sites and MTS.

    n_atomistic chains of nmono monomers, each monomer 4 backbone carbons in a
    112-degree zig-zag with 2 hydrogens per carbon (12 atoms, label A) and one
    virtual site at its centre of mass; n_cg chains of nmono explicit CG beads
    (label B), one per monomer.  Chains run straight along x on a 0.65 nm grid
    in y and z; the box is one chain length plus a gap in x.  Atom-atom tables
    (C, H) to 1.0 nm (list 1.2 nm), bead/site tables to 1.4 nm (list 1.6 nm) as a
    smooth seeded IBI-like potential: LJ plus Fourier modes.  The reference
    pairs atoms only with atoms, and beads with beads and sites, but never sites
    with sites, so the CG chains are what the site tables act on.  MTS evaluates
    the CG nonbonded forces on 3 of every 3 + nmts steps; bonded terms and atom
    nonbonded run every step.  Berendsen NVT, dt 1 fs."""
    rng = np.random.default_rng(seed)
    bond, theta = 0.155, np.radians(112.0)
    dx, dy = bond * np.sin(theta / 2), bond * np.cos(theta / 2)   # zig-zag step along x, offset in y
    mono_len = 4 * dx
    cg_bond = mono_len / np.sin(np.radians(75.0))
    cg_dy = cg_bond * np.cos(np.radians(75.0))
    grid = 0.65
    nrow = n_atomistic + n_cg
    ny = int(np.ceil(np.sqrt(nrow)))
    nz = int(np.ceil(nrow / ny))
    box = (nmono * mono_len + 0.5, ny * grid, nz * grid)
    types = [("C", 0.012, "A"), ("H", 0.001008, "A"), ("B", 0.170, "B"), ("V", 0.170, "B")]
    pos, itype, bonds, mols, virt = [], [], [], [], []
    alpha = np.radians(54.75)
    for ch in range(n_atomistic):
        y0 = -0.5 * box[1] + (ch % ny + 0.5) * grid
        z0 = -0.5 * box[2] + (ch // ny + 0.5) * grid
        first = len(pos)
        nc = 4 * nmono
        cids = []
        for k in range(nc):
            cids.append(len(pos))
            pos.append((-0.5 * box[0] + 0.25 + k * dx, y0 + (k % 2) * dy, z0))
            itype.append(1)
            bonds.append([])
        for k in range(nc):
            c = np.array(pos[cids[k]])
            away = np.array([0.0, -1.0 if k % 2 == 0 else 1.0, 0.0])
            for sgn in (1.0, -1.0):
                h = c + bond * 0.7 * (np.cos(alpha) * away + sgn * np.sin(alpha) * np.array([0.0, 0.0, 1.0]))
                hid = len(pos)
                pos.append(tuple(h))
                itype.append(2)
                bonds.append([cids[k] + 1])
                bonds[cids[k]].append(hid + 1)
        for k in range(nc - 1):
            bonds[cids[k]].append(cids[k + 1] + 1)
            bonds[cids[k + 1]].append(cids[k] + 1)
        # molecule = chain; a site per monomer at the centre of mass of its 12 atoms
        mols.append(("achain", len(pos) - first))
        for m in range(nmono):
            members = []
            for k in range(4 * m, 4 * m + 4):
                members.append(cids[k] + 1)
                members.extend(b for b in bonds[cids[k]] if itype[b - 1] == 2)
            virt.append((4, sorted(members), 0))
    # the reference lists a particle's bonded partners in coordinate-file order
    for ch in range(n_cg):
        row = n_atomistic + ch
        y0 = -0.5 * box[1] + (row % ny + 0.5) * grid
        z0 = -0.5 * box[2] + (row // ny + 0.5) * grid
        first = len(pos)
        for m in range(nmono):  # a 150-degree zig-zag (a straight angle has no plane)
            pos.append((-0.5 * box[0] + 0.25 + (m + 0.5) * mono_len, y0 + (m % 2) * cg_dy, z0))
            itype.append(3)
            nb = []
            if m > 0:
                nb.append(first + m)
            if m < nmono - 1:
                nb.append(first + m + 2)
            bonds.append(nb)
        mols.append(("cgchain", nmono))
    pos = np.array(pos)
    natoms = len(pos)
    masses = [types[t - 1][1] for t in itype]
    vel = maxwell_boltzmann(rng, masses, temp)
    control = dict(ensemble="NVT", temperature=temp, pressure=101.3, atoms=natoms, num_of_time_steps=nsteps,
                   time_step=0.001, temperature_coupling_time="0.1D0", pressure_coupling_time="1.0D0",
                   isothermal_compressibility="4.5D-5", virtual_sites=len(virt), mts=nmts, bead_cutoff=1.4,
                   bead_neighbour_list_cutoff=1.6, non_bonded_bead=4, cutoff=1.0, neighbour_list_cutoff=1.2,
                   update_neighbour_list=10, trajectory=nsteps, halt_drift=nsteps + 1, non_bonded=4,
                   initialize_velocities="N")
    cc = harmonic_bond_table("bcc.tab", bond, 2.5e5, 0.6, 0.0003)
    ch_t = harmonic_bond_table("bch.tab", bond * 0.7, 2.5e5, 0.6, 0.0003)
    bb = harmonic_bond_table("bbb.tab", cg_bond, 5.0e3, 1.2, 0.001)
    ang = harmonic_angle_table("ang.tab", 112.0, 400.0)
    ang_cg = harmonic_angle_table("angcg.tab", 150.0, 20.0)
    tor = cosine_torsion_table("tors.tab", 5.0)
    sig = {(1, 1): 0.34, (1, 2): 0.29, (2, 2): 0.24}
    eps = {(1, 1): 0.35, (1, 2): 0.15, (2, 2): 0.06}
    nb = [(k, lj_table(f"nba{k[0]}{k[1]}", sig[k], eps[k], 1.0, 0.002)) for k in sorted(sig)]
    for k in ((3, 3), (3, 4), (4, 4)):
        amps = rng.uniform(-0.5, 0.5, size=5) / 5.0
        nb.append((k, perturbed_lj_table(f"nbc{k[0]}{k[1]}", 0.5, 1.0, 1.4, 0.002, amps)))
    return SystemSpec(
        control=control, types=types, pos=pos, vel=vel, itype=np.array(itype), bonds=bonds, molecules=mols,
        box=box, bond_tabs=[((1, 1), cc), ((1, 2), ch_t), ((3, 3), bb)],
        angle_tabs=[((1, 1, 1), ang), ((1, 1, 2), ang), ((2, 1, 2), ang), ((3, 3, 3), ang_cg)],
        torsion_tabs=[((1, 1, 1, 1), tor)],
        nb_tabs=nb, virtual=virt)


# ------------------------------------------------------------ served jobs
def serpentine_lattice(m):
    """The m^3 sites of a cubic lattice in an order where consecutive sites
    are nearest neighbours (boustrophedon in x, then y, then z)."""
    pts = []
    for z in range(m):
        ys = range(m) if z % 2 == 0 else range(m - 1, -1, -1)
        for j, y in enumerate(ys):
            xs = range(m) if (z * m + j) % 2 == 0 else range(m - 1, -1, -1)
            for x in xs:
                pts.append((x, y, z))
    return np.asarray(pts, float)


def serving_job(seed, n_target, rho=8.0, nsteps=2000, temp=300.0, amp=0.5):
    """One job of a served stream: bead-spring chains of 10-100 beads with 1-3
    bead types, placed along a serpentine path through a cubic lattice of
    spacing rho^(-1/3) (bonds at their rest length, no overlaps), each type
    pair with its own LJ table plus a seeded smooth perturbation of 5 Fourier
    modes (amplitudes up to amp kJ/mol).  rc 1.0 nm, list 1.2 nm every 10 steps,
    NVT at temp, dt 10 fs."""
    rng = np.random.default_rng(seed)
    nper = int(rng.integers(10, 101))
    nchains = max(1, int(round(n_target / nper)))
    n = nchains * nper
    a = rho ** (-1.0 / 3.0)
    m = int(np.ceil(n ** (1.0 / 3.0)))
    box = m * a
    pos = serpentine_lattice(m)[:n] * a - 0.5 * box + 0.5 * a
    pos += rng.normal(scale=0.01, size=pos.shape)
    ntypes = int(rng.integers(1, 4))
    types = list(range(1, ntypes + 1))
    itype = np.array([1 + (k % ntypes) for ch in range(nchains) for k in range(nper)])
    mass = 0.072
    vel = maxwell_boltzmann(rng, [mass] * n, temp)
    bond_t = harmonic_bond_table("bond.tab", a, 5.0e3, 1.0, 0.001)
    nb = []
    for i in types:
        for j in types:
            if i <= j:
                amps = rng.uniform(-amp, amp, size=5) / 5.0
                nb.append(((i, j), perturbed_lj_table(f"nb{i}{j}", 0.47, 3.5, 1.0, 0.002, amps)))
    control = dict(ensemble="NVT", temperature=temp, pressure=101.3, atoms=n, num_of_time_steps=nsteps,
                   time_step=0.010, temperature_coupling_time="0.1D0", pressure_coupling_time="5.0D0",
                   isothermal_compressibility="1.0D-6", virtual_sites=0, mts=0, bead_cutoff=1.0,
                   bead_neighbour_list_cutoff=1.2, non_bonded_bead=4, cutoff=1.0, neighbour_list_cutoff=1.2,
                   update_neighbour_list=10, trajectory=nsteps, halt_drift=nsteps + 1, non_bonded=4,
                   initialize_velocities="N")
    return SystemSpec(control=control, types=[(f"C{t}", mass, "A") for t in types], pos=pos, vel=vel,
                      itype=itype, bonds=chain_bonds(nchains, nper), molecules=[("chain", nper)] * nchains,
                      box=(box, box, box), bond_tabs=[((i, j), bond_t) for i in types for j in types if i <= j],
                      nb_tabs=nb)


def job_stream(njobs, seed=5, nmin=500, nmax=50000, rate=20.0):
    """Sizes log-uniform in [nmin, nmax] and Poisson arrival times (jobs/s) of
    a served stream: [(arrival_s, n_target, job_seed)]."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=njobs)).astype(int)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=njobs))
    arrivals -= arrivals[0]
    return [(float(t), int(nn), int(seed * 100003 + k)) for k, (t, nn) in enumerate(zip(arrivals, sizes))]
