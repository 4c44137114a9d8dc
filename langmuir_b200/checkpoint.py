"""Langmuir checkpoint files (.chk, .chk.gz) for the GPU kMC.

The reference's CheckPointer (src/langmuirCore/checkpointer.cpp) writes the
sections [Electrons], [Holes], [Defects], [Traps], optionally
[TrapPotentials], [FluxState], [RandomState] and [Parameters]; each list
section is a count followed by that many values (checkpointer.cpp:213-548).
``read`` parses the same format and ``write`` produces it from a running
replica.  ``resume`` builds a replica from a checkpoint with
``lgm_kmc_create_from``, which places the listed sites before drawing the rest
(World::initialize, world.cpp:619-657).

The random state is the one difference.  The reference serialises its Boost
mt19937; this library draws from a counter-based Philox stream keyed by
(random.seed, replica) and the step.  A checkpoint therefore needs no
generator state: resumed with the same random.seed and replica at
current.step, the run continues exactly where it stopped.  ``read`` accepts
and skips a [RandomState] section, and ``write`` omits it, which makes the
reference reseed from random.seed when it reads the file.
"""
from __future__ import annotations

import gzip
from dataclasses import dataclass, field

import numpy as np

from .kmc import KMC, Params

SECTIONS = ("Parameters", "Electrons", "Holes", "Defects", "Traps", "TrapPotentials",
            "RandomState", "FluxState")

# this library's counters (eSL eSR hSL hSR eDL eDR hDL hDR xSource xDrain, each
# attempts/successes) -> the reference's flux-agent order (world.cpp:961-1187):
# eSL eSR hSL hSR xSource eDL eDR hDL hDR xDrain
FLUX_ORDER = (0, 1, 2, 3, 8, 4, 5, 6, 7, 9)
FLUX_NAMES = ("eSourceL", "eSourceR", "hSourceL", "hSourceR", "xSource", "eDrainL", "eDrainR",
              "hDrainL", "hDrainR", "xDrain")


def reference_flux(counters) -> list:
    """Our 20 counters in the reference's [FluxState] / out.dat order."""
    c = list(counters)
    out = []
    for agent in FLUX_ORDER:
        out += [int(c[2 * agent]), int(c[2 * agent + 1])]
    return out


@dataclass
class Checkpoint:
    params: Params
    electrons: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    holes: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    defects: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    traps: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    trap_potentials: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    flux: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint64))
    had_random_state: bool = False

    def world(self) -> dict:
        return dict(electrons=self.electrons, holes=self.holes, defects=self.defects,
                    traps=self.traps, trap_potentials=self.trap_potentials, flux=self.flux)


def _text(path_or_text: str) -> str:
    if "\n" in path_or_text or path_or_text.lstrip().startswith("["):
        return path_or_text
    if path_or_text.endswith(".gz"):
        with gzip.open(path_or_text, "rt") as fh:
            return fh.read()
    with open(path_or_text) as fh:
        return fh.read()


def read(path_or_text: str, params: Params | None = None) -> Checkpoint:
    """Parse a checkpoint (a file name, .gz allowed, or its text).  Section
    names and their order follow CheckPointer::load (checkpointer.cpp:22-163):
    any order, each at most once in practice; [Parameters] runs to a line
    "end" or to the end of the text; an unknown section is an error."""
    text = _text(path_or_text)
    lines = text.split("\n")
    ck = Checkpoint(params=params if params is not None else Params.default())
    i = 0
    tokens: list[str] = []

    def take_tokens(start):
        """Whitespace-separated tokens from line `start` up to the next section."""
        out, j = [], start
        while j < len(lines) and not lines[j].strip().startswith("["):
            out += lines[j].split()
            j += 1
        return out, j

    while i < len(lines):
        line = lines[i].strip()
        if not line:
            i += 1
            continue
        if not line.startswith("["):
            raise ValueError(f"langmuir: expected a section header or empty line, got {line!r}")
        name = line.replace("[", "").replace("]", "").strip()
        if name not in SECTIONS:
            raise ValueError(f"langmuir: invalid section encountered: {name}; valid sections are "
                             + ", ".join(f"[{s}]" for s in SECTIONS))
        if name == "Parameters":
            j = i + 1
            body = []
            while j < len(lines):
                if lines[j].strip().lower() == "end":
                    j += 1
                    break
                if lines[j].strip().startswith("[") and lines[j].strip().strip("[]") in SECTIONS:
                    break
                body.append(lines[j])
                j += 1
            ck.params.parse("[Parameters]\n" + "\n".join(body) + "\n")
            i = j
            continue
        tokens, j = take_tokens(i + 1)
        if name == "RandomState":
            ck.had_random_state = True
            i = j
            continue
        if not tokens:
            raise ValueError(f"langmuir: stream error: expected the number of values of [{name}]")
        n = int(tokens[0])
        vals = tokens[1:1 + n]
        if len(vals) != n:
            raise ValueError(f"langmuir: stream error: [{name}] lists {len(vals)} of {n} values")
        if name == "TrapPotentials":
            setattr(ck, "trap_potentials", np.array([float(v) for v in vals], np.float64))
        elif name == "FluxState":
            ck.flux = np.array([int(v) for v in vals], np.uint64)
        else:
            setattr(ck, name.lower(), np.array([int(v) for v in vals], np.int32))
        i = j
    return ck


def write(kmc: KMC, trap_potentials: bool | None = None) -> str:
    """Checkpoint text of a replica, sections in CheckPointer::save order
    (checkpointer.cpp:165-193): carriers in list order, defects, traps,
    [TrapPotentials] when output.chk.trap.potential is set (or asked for),
    [FluxState] in the reference's flux-agent order, and [Parameters] with
    current.step at the replica's step.  No [RandomState] (see the module
    docstring)."""
    s = kmc.stats()
    e, h = kmc.carriers()
    w = kmc.world()
    p = Params()
    ctypes_copy(kmc.params, p)
    p.current_step = s["step"]
    want_tp = bool(p.output_chk_trap_potential) if trap_potentials is None else trap_potentials

    def section(name, values, fmt=str):
        return "\n".join([f"[{name}]", str(len(values))] + [fmt(v) for v in values])

    parts = [section("Electrons", e), section("Holes", h), section("Defects", w["defects"]),
             section("Traps", w["traps"])]
    if want_tp:
        # saveTrapPotentials: scientific with digits10 + 2 = 17 digits
        parts.append(section("TrapPotentials", w["trap_potentials"], lambda v: f"{v:.17e}"))
    parts.append(section("FluxState", reference_flux(s["counters"])))
    return "\n".join(parts) + "\n" + p.format()


def ctypes_copy(src, dst):
    import ctypes
    ctypes.memmove(ctypes.byref(dst), ctypes.byref(src), ctypes.sizeof(src))


def save(kmc: KMC, path: str, **kw) -> None:
    text = write(kmc, **kw)
    if path.endswith(".gz"):
        with gzip.open(path, "wt") as fh:
            fh.write(text)
    else:
        with open(path, "w") as fh:
            fh.write(text)


def resume(path_or_text: str, device: int = 0, replica: int = 0,
           params: Params | None = None) -> KMC:
    """A replica built from a checkpoint: its parameters (current.step
    included), and its listed carriers, defects, traps and flux counters."""
    ck = read(path_or_text, params)
    return KMC(ck.params.check(), device=device, replica=replica, world=ck.world())
