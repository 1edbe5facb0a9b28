"""Seeded synthetic molecules in libcint's (atm, bas, env) format.

The five workloads of this engine are synthetic: a 3-atom water-like molecule, a 40-atom
s/p/d molecule, a 120-atom s/p/d/f molecule, a 20-atom molecule with g shells and a
density-fitting auxiliary basis on the 120-atom molecule.  They are built here with a
self-contained splitmix64 generator so that every platform (this host, the GPU host, C
drivers) sees bit-identical inputs for a given seed.

Array layout follows libcint's `cint.h.in`:
  atm[natm, 6]  = (charge, ptr_coord, nuc_mod, ptr_zeta, ptr_frac_charge, reserved)
  bas[nbas, 8]  = (atom_of, ang_of, nprim_of, nctr_of, kappa_of, ptr_exp, ptr_coeff, reserved)
  env[...]      = global slots 0..19 (PTR_ENV_START = 20), then coordinates, exponents and
                  column-major contraction coefficients (coeff[ctr * nprim + prim]).
Contraction coefficients are multiplied by the radial GTO norm (libcint `CINTgto_norm`,
`libcint-master/src/misc.c:86`) and the contracted shell is renormalised to unit radial
self-overlap, which is what libcint callers (PySCF `make_bas_env`) store in env.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# libcint slot constants (libcint-master/include/cint.h.in:28-66)
PTR_EXPCUTOFF = 0
PTR_RANGE_OMEGA = 8
PTR_ENV_START = 20
ATM_SLOTS = 6
BAS_SLOTS = 8
CHARGE_OF, PTR_COORD, NUC_MOD_OF, PTR_ZETA = 0, 1, 2, 3
ATOM_OF, ANG_OF, NPRIM_OF, NCTR_OF, KAPPA_OF, PTR_EXP, PTR_COEFF = 0, 1, 2, 3, 4, 5, 6

EXP_LO, EXP_HI = 0.1, 1.2e4


class SplitMix64:
    """splitmix64 stream (Steele, Lea & Flood 2014); uniform doubles use the top 53 bits."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.state = seed & self.MASK

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & self.MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        u = (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)
        return lo + (hi - lo) * u

    def log_uniform(self, lo: float, hi: float) -> float:
        return math.exp(self.uniform(math.log(lo), math.log(hi)))

    def normal(self) -> float:
        # Box-Muller; u1 in (0, 1] so the log is finite
        u1 = 1.0 - self.uniform()
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def gaussian_int(n: int, alpha: float) -> float:
    """int_0^inf r^n exp(-alpha r^2) dr (libcint `_gaussian_int`, misc.c:72)."""
    n1 = (n + 1) * 0.5
    return math.exp(math.lgamma(n1)) / (2.0 * alpha ** n1)


def gto_norm(l: int, a: float) -> float:
    """Radial norm of r^l exp(-a r^2) (libcint `CINTgto_norm`, misc.c:86)."""
    return 1.0 / math.sqrt(gaussian_int(2 * l + 2, 2 * a))


@dataclass
class ShellSpec:
    l: int
    exps: list
    coeffs: list  # one contraction (nctr = 1)


@dataclass
class Molecule:
    name: str
    atm: np.ndarray
    bas: np.ndarray
    env: np.ndarray
    coords: np.ndarray
    shell_atoms: list = field(default_factory=list)

    @property
    def natm(self) -> int:
        return self.atm.shape[0]

    @property
    def nbas(self) -> int:
        return self.bas.shape[0]

    def shell_l(self, i: int) -> int:
        return int(self.bas[i, ANG_OF])

    def nsph(self, i: int) -> int:
        return (2 * int(self.bas[i, ANG_OF]) + 1) * int(self.bas[i, NCTR_OF])

    def ncart(self, i: int) -> int:
        l = int(self.bas[i, ANG_OF])
        return (l + 1) * (l + 2) // 2 * int(self.bas[i, NCTR_OF])

    def ao_loc(self, cart: bool = False) -> np.ndarray:
        f = self.ncart if cart else self.nsph
        loc = np.zeros(self.nbas + 1, dtype=np.int64)
        for i in range(self.nbas):
            loc[i + 1] = loc[i] + f(i)
        return loc


def make_shell(rng: SplitMix64, l: int, nprim: int) -> ShellSpec:
    exps = sorted((rng.log_uniform(EXP_LO, EXP_HI) for _ in range(nprim)), reverse=True)
    raw = [rng.normal() for _ in range(nprim)]
    if nprim == 1:
        raw = [1.0]  # a single primitive has no freedom after renormalisation except sign
    cs = [c * gto_norm(l, a) for c, a in zip(raw, exps)]
    # contracted radial self-overlap: sum_pq c_p c_q int r^(2l+2) exp(-(a_p+a_q) r^2)
    s = 0.0
    for p in range(nprim):
        for q in range(nprim):
            s += cs[p] * cs[q] * gaussian_int(2 * l + 2, exps[p] + exps[q])
    nrm = 1.0 / math.sqrt(s)
    return ShellSpec(l, exps, [c * nrm for c in cs])


def build_molecule(name: str, coords, atom_shells) -> Molecule:
    """Pack per-atom shell lists into libcint atm/bas/env arrays."""
    env = [0.0] * PTR_ENV_START
    atm = []
    for xyz in coords:
        ptr = len(env)
        env.extend(float(v) for v in xyz)
        atm.append([1, ptr, 1, 0, 0, 0])
    bas = []
    shell_atoms = []
    for ia, shells in enumerate(atom_shells):
        for sh in shells:
            pexp = len(env)
            env.extend(sh.exps)
            pcoef = len(env)
            env.extend(sh.coeffs)
            bas.append([ia, sh.l, len(sh.exps), 1, 0, pexp, pcoef, 0])
            shell_atoms.append(ia)
    return Molecule(
        name=name,
        atm=np.asarray(atm, dtype=np.int32).reshape(-1, ATM_SLOTS),
        bas=np.asarray(bas, dtype=np.int32).reshape(-1, BAS_SLOTS),
        env=np.asarray(env, dtype=np.float64),
        coords=np.asarray(coords, dtype=np.float64).reshape(-1, 3),
        shell_atoms=shell_atoms,
    )


# (l, nprim) per shell of each atom kind
HEAVY = [(0, 8), (0, 8), (0, 1), (1, 3), (1, 1), (2, 1)]
HEAVY_F = HEAVY + [(3, 1)]
LIGHT = [(0, 3), (0, 1), (1, 1)]
G_ATOM = [(0, 3), (1, 1), (2, 1), (4, 1)]
AUX = [(0, 1)] * 6 + [(1, 1)] * 5 + [(2, 1)] * 4 + [(3, 1)] * 3 + [(4, 1)] * 2


def _place_atoms(rng: SplitMix64, natm: int, box: float, min_sep: float):
    coords = []
    while len(coords) < natm:
        p = [rng.uniform(-0.5 * box, 0.5 * box) for _ in range(3)]
        if all(sum((a - b) ** 2 for a, b in zip(p, q)) >= min_sep ** 2 for q in coords):
            coords.append(p)
    return coords


def _kinds(rng: SplitMix64, natm: int, frac_light: float):
    nlight = int(round(frac_light * natm))
    kinds = ["light"] * nlight + ["heavy"] * (natm - nlight)
    for i in range(natm - 1, 0, -1):  # Fisher-Yates with the same stream
        j = rng.next_u64() % (i + 1)
        kinds[i], kinds[j] = kinds[j], kinds[i]
    return kinds


def water_like(seed: int = 0) -> Molecule:
    """3 atoms: O at the origin, two H at 1.8 bohr, 104.5 degrees apart."""
    rng = SplitMix64(seed)
    half = math.radians(104.5) / 2
    coords = [[0.0, 0.0, 0.0],
              [1.8 * math.sin(half), 0.0, 1.8 * math.cos(half)],
              [-1.8 * math.sin(half), 0.0, 1.8 * math.cos(half)]]
    shells = [[make_shell(rng, l, n) for l, n in HEAVY]]
    shells += [[make_shell(rng, l, n) for l, n in LIGHT] for _ in range(2)]
    return build_molecule("water3", coords, shells)


def random_molecule(name: str, seed: int, natm: int, box: float, with_f: bool,
                    frac_light: float = 0.6, min_sep: float = 1.4) -> Molecule:
    rng = SplitMix64(seed)
    coords = _place_atoms(rng, natm, box, min_sep)
    kinds = _kinds(rng, natm, frac_light)
    heavy = HEAVY_F if with_f else HEAVY
    shells = [[make_shell(rng, l, n) for l, n in (LIGHT if k == "light" else heavy)]
              for k in kinds]
    return build_molecule(name, coords, shells)


def mol40(seed: int = 1) -> Molecule:
    return random_molecule("mol40_spd", seed, 40, 14.0, with_f=False)


def mol120(seed: int = 2) -> Molecule:
    return random_molecule("mol120_spdf", seed, 120, 22.0, with_f=True)


def mol20_g(seed: int = 3) -> Molecule:
    rng = SplitMix64(seed)
    coords = _place_atoms(rng, 20, 12.0, 1.4)
    shells = [[make_shell(rng, l, n) for l, n in G_ATOM] for _ in range(20)]
    return build_molecule("mol20_g", coords, shells)


def with_aux(mol: Molecule, seed: int = 4, exp_lo: float = 0.05, exp_hi: float = 5e3) -> Molecule:
    """Append a per-atom auxiliary basis (6s 5p 4d 3f 2g single primitives) to `mol`.

    Auxiliary shells follow the orbital shells in `bas`; `mol.nbas` orbital shells come first.
    """
    rng = SplitMix64(seed)
    env = list(mol.env)
    bas = [list(r) for r in mol.bas]
    for ia in range(mol.natm):
        for l, _ in AUX:
            a = rng.log_uniform(exp_lo, exp_hi)
            pexp = len(env)
            env.append(a)
            pcoef = len(env)
            env.append(gto_norm(l, a))
            bas.append([ia, l, 1, 1, 0, pexp, pcoef, 0])
    return Molecule(name=mol.name + "+aux", atm=mol.atm.copy(),
                    bas=np.asarray(bas, dtype=np.int32), env=np.asarray(env),
                    coords=mol.coords.copy(),
                    shell_atoms=[int(b[0]) for b in bas])


CONFIGS = {
    "water3": water_like,
    "mol40_spd": mol40,
    "mol120_spdf": mol120,
    "mol20_g": mol20_g,
}
