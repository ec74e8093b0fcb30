"""Seeded synthetic potential-energy surfaces (PES) in the reference input format.

The reference program reads a positional text file (`src/Input_Reader.cpp:170-246`):

    Comment line
    HCI_Eps: <eps1>
    Nstate: <k>
    PT2: <0|1>
    PT2_Eps: <eps2>
    Max_quanta: <Ntot>
    Modes: <Nm>
     <id> <freq> <cap>
    Force_constants: <Nfc>
     <order> <mode> ... <mode> <value>

This module writes such files for the benchmark workloads, so that the CPU oracle, the reference
binary and the GPU build all read one identical file.  Every draw comes from one
`numpy.random.Generator(PCG64(seed))` stream in a fixed order:

* harmonic frequencies: Nm draws of U[500, 3300] cm^-1, sorted ascending; per-mode cap 8;
* cubic terms: for every multiset i<=j<=k in lexicographic order, keep with probability p3,
  value s * 10^U(a3, b3) with a random sign s;
* quartic terms: every multiset i<=j<=k<=l, keep with p4, value s * 10^U(a4, b4); the diagonal
  iiii terms are positive;
* optional quintic terms (all multisets, keep p5, random sign) and sextic "diagonal/pair" terms
  (multisets with at most two distinct modes, i^6 and i^a j^(6-a), keep p6, positive).

Values are written with 10 decimals, so every reader parses the same doubles.

Admissibility.  Independent random cubic/quartic terms often make the potential fall below its
expansion minimum a few quanta out (e.g. a large cubic term on a soft mode with no diagonal
quartic).  Heat-bath selection then walks into that region and the variational energy collapses
without converging — the reference procedure does the same on such a surface.  A workload
therefore uses the first draw, over seeds base + 100*j (j = 0, 1, ...), whose potential is
non-negative on every one- and two-mode plane within |q| <= sqrt(2*16+1) and on every three-mode
cube within |q| <= sqrt(2*12+1) (dimensionless normal coordinates, V = sum w q^2/2 +
sum phi/prod(p_k!) prod q^p_k, i.e. the region spanned by up to 16 resp. 12 quanta per mode).
`admissible()` implements the test and `WORKLOAD_SEED_OFFSET` records the first accepted j.
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field

import numpy as np

SEED_BASE = 20260000


@dataclass
class PESSpec:
    nmodes: int
    p3: float = 0.5
    r3: tuple = (0.0, 2.5)
    p4: float = 0.3
    r4: tuple = (-1.0, 1.5)
    p5: float = 0.0
    r5: tuple = (-2.0, 0.5)
    p6: float = 0.0
    r6: tuple = (-2.0, 0.5)
    freq_range: tuple = (500.0, 3300.0)
    cap: int = 8


@dataclass
class RunSettings:
    eps1: float
    nstate: int
    pt2: int
    eps2: float
    ntot: int = 2


@dataclass
class PES:
    freqs: list
    caps: list
    fcs: list = field(default_factory=list)  # list of (modes tuple, value)


def generate(spec: PESSpec, seed: int) -> PES:
    rng = np.random.Generator(np.random.PCG64(seed))
    nm = spec.nmodes
    freqs = sorted(float(x) for x in rng.uniform(spec.freq_range[0], spec.freq_range[1], nm))
    freqs = [float("%.6f" % f) for f in freqs]
    pes = PES(freqs=freqs, caps=[spec.cap] * nm)

    def draw(order, p, rng_range, positive_rule, subset=None):
        for ms in itertools.combinations_with_replacement(range(nm), order):
            if subset is not None and not subset(ms):
                continue
            keep = rng.random() < p
            mag = 10.0 ** rng.uniform(rng_range[0], rng_range[1])
            sgn = -1.0 if rng.random() < 0.5 else 1.0
            if not keep:
                continue
            if positive_rule(ms):
                sgn = 1.0
            pes.fcs.append((ms, sgn * mag))

    if spec.p3 > 0:
        draw(3, spec.p3, spec.r3, lambda ms: False)
    if spec.p4 > 0:
        draw(4, spec.p4, spec.r4, lambda ms: len(set(ms)) == 1)
    if spec.p5 > 0:
        draw(5, spec.p5, spec.r5, lambda ms: False)
    if spec.p6 > 0:
        draw(6, spec.p6, spec.r6, lambda ms: True, subset=lambda ms: len(set(ms)) <= 2)
    return pes


def write_input(path: str, pes: PES, run: RunSettings, comment: str = "synthetic PES") -> None:
    lines = [f"Comment: {comment}",
             f"HCI_Eps: {run.eps1!r}",
             f"Nstate: {run.nstate}",
             f"PT2: {run.pt2}",
             f"PT2_Eps: {run.eps2!r}",
             f"Max_quanta: {run.ntot}",
             f"Modes: {len(pes.freqs)}"]
    for i, (f, c) in enumerate(zip(pes.freqs, pes.caps)):
        lines.append(f" {i} {f:.6f} {c}")
    lines.append(f"Force_constants: {len(pes.fcs)}")
    for ms, v in pes.fcs:
        lines.append(" %d %s %.10f" % (len(ms), " ".join(str(m) for m in ms), v))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


# Benchmark workloads (mode counts, keep probabilities, value ranges and run settings).
WORKLOADS = {
    0: (PESSpec(12), RunSettings(eps1=1.0, nstate=50, pt2=0, eps2=0.0)),
    1: (PESSpec(15), RunSettings(eps1=0.5, nstate=200, pt2=1, eps2=0.01)),
    2: (PESSpec(48, p3=0.15, p4=0.02), RunSettings(eps1=1.0, nstate=128, pt2=1, eps2=0.2)),
    4: (PESSpec(30, p3=0.3, p4=0.1, p5=0.01, p6=0.05),
        RunSettings(eps1=0.1, nstate=100, pt2=1, eps2=0.05)),
}


# First admissible draw j (seed = base + 100*j) per workload, found with `find_admissible`.
WORKLOAD_SEED_OFFSET = {0: 0, 1: 1, 2: 39, 4: 6}


def base_seed(workload: int, request: int = 0) -> int:
    return SEED_BASE + workload * 1000 + request


def workload_seed(workload: int) -> int:
    return base_seed(workload) + 100 * WORKLOAD_SEED_OFFSET.get(workload, 0)


def _subset_terms(pes: PES):
    """FC terms keyed by their mode set: list of (modes, powers, coefficient / prod p!)."""
    from math import factorial
    out = {}
    for ms, v in pes.fcs:
        modes = tuple(sorted(set(ms)))
        pw = tuple(ms.count(m) for m in modes)
        den = 1.0
        for p in pw:
            den *= factorial(p)
        out.setdefault(modes, []).append((modes, pw, v / den))
    return out


def _min_potential(pes: PES, terms, modes, qmax, ng):
    g = np.linspace(-qmax, qmax, ng)
    grids = np.meshgrid(*([g] * len(modes)), indexing="ij")
    q = {m: grids[i].ravel() for i, m in enumerate(modes)}
    V = np.zeros(grids[0].size)
    for m in modes:
        V += 0.5 * pes.freqs[m] * q[m] ** 2
    for r in range(1, len(modes) + 1):
        for sub in itertools.combinations(modes, r):
            for tm, pw, c in terms.get(sub, ()):
                t = np.full(V.shape, c)
                for m, p in zip(tm, pw):
                    t = t * q[m] ** p
                V += t
    return float(V.min())


def admissible(pes: PES, pair_quanta: int = 16, triple_quanta: int = 12) -> bool:
    """Potential >= 0 on all one/two-mode planes and three-mode cubes of the stated extent."""
    terms = _subset_terms(pes)
    nm = len(pes.freqs)
    q2 = math.sqrt(2 * pair_quanta + 1)
    q3 = math.sqrt(2 * triple_quanta + 1)
    for i, j in itertools.combinations(range(nm), 2):
        if _min_potential(pes, terms, (i, j), q2, 41) < 0:
            return False
    for tri in itertools.combinations(range(nm), 3):
        if _min_potential(pes, terms, tri, q3, 13) < 0:
            return False
    return True


def find_admissible(workload: int, max_tries: int = 50) -> int:
    spec, _ = WORKLOADS[workload]
    for j in range(max_tries):
        if admissible(generate(spec, base_seed(workload) + 100 * j)):
            return j
    raise RuntimeError(f"no admissible draw for workload {workload} in {max_tries} tries")


def write_workload(path: str, workload: int, run: RunSettings | None = None) -> None:
    spec, default_run = WORKLOADS[workload]
    pes = generate(spec, workload_seed(workload))
    write_input(path, pes, run or default_run, comment=f"synthetic PES, workload {workload}")


def serving_request(request: int):
    """One request of the mixed serving stream: Nm in {6..24}, Nstate in {10..100}, eps1 log-uniform
    in [0.3, 3], PT2 on with eps2 = 0.1 * eps1.  The settings come from the request's own stream;
    the PES is redrawn (seed + 100000 j) until it passes `admissible`.  Returns (PES, RunSettings)."""
    rng = np.random.Generator(np.random.PCG64(base_seed(3, request) + 500))
    nm = int(rng.integers(6, 25))
    nstate = int(rng.integers(10, 101))
    eps1 = float("%.6f" % math.exp(rng.uniform(math.log(0.3), math.log(3.0))))
    eps2 = float("%.6f" % (0.1 * eps1))
    for j in range(200):
        pes = generate(PESSpec(nm), base_seed(3, request) + 100000 * j)
        if admissible(pes):
            return pes, RunSettings(eps1=eps1, nstate=nstate, pt2=1, eps2=eps2)
    raise RuntimeError(f"no admissible PES for serving request {request}")
