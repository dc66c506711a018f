"""Seeded synthetic water structures (the benchmark and test workloads).

Rigid water molecules (O-H 1.81 bohr, H-O-H 104.5 deg) at density
1.0 g/cm^3 in a periodic cubic box, oxygens placed uniformly at random with an
O-O >= 4.7 bohr minimum-image rejection, orientations uniform.  Atoms are
listed O, H, H per molecule.  Element indices follow n2p2's element order
(sorted by atomic number): H = 0, O = 1.
"""
from __future__ import annotations

import math

import numpy as np

BOHR_CM = 0.529177210903e-8
AVOGADRO = 6.02214076e23
M_WATER = 18.01528          # g/mol
OH_BOHR = 1.81
HOH_DEG = 104.5
MIN_OO_BOHR = 4.7
H, O = 0, 1


def molecules_per_bohr3(density_g_cm3: float = 1.0) -> float:
    return density_g_cm3 * AVOGADRO / M_WATER * BOHR_CM ** 3


def box_length(n_molecules: int, density_g_cm3: float = 1.0) -> float:
    return (n_molecules / molecules_per_bohr3(density_g_cm3)) ** (1.0 / 3.0)


def _place_oxygens(n: int, L: float, rng: np.random.Generator,
                   min_oo: float) -> np.ndarray:
    """Random sequential addition with a cell grid (minimum image)."""
    nc = max(1, int(L // min_oo))
    cw = L / nc
    grid: dict = {}
    out = np.zeros((n, 3))
    placed = 0
    min2 = min_oo * min_oo
    attempts = 0
    batch = 256
    while placed < n:
        cand = rng.uniform(0.0, L, size=(batch, 3))
        for p in cand:
            attempts += 1
            if attempts > 500 * n + 100000:
                raise RuntimeError("water placement did not converge")
            c = np.floor(p / cw).astype(int) % nc
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        key = ((c[0] + dx) % nc, (c[1] + dy) % nc,
                               (c[2] + dz) % nc)
                        for q in grid.get(key, ()):
                            d = p - out[q]
                            d -= L * np.round(d / L)
                            if d @ d < min2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                out[placed] = p
                grid.setdefault((c[0], c[1], c[2]), []).append(placed)
                placed += 1
                if placed == n:
                    break
    return out


def water_box(n_molecules: int, seed: int, density: float = 1.0,
              min_oo: float = MIN_OO_BOHR):
    """(box[3,3], positions[3n,3], elements[3n]) for one water box."""
    rng = np.random.default_rng(seed)
    L = box_length(n_molecules, density)
    ox = _place_oxygens(n_molecules, L, rng, min_oo)
    u = rng.normal(size=(n_molecules, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = rng.normal(size=(n_molecules, 3))
    v -= (v * u).sum(axis=1, keepdims=True) * u
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    th = math.radians(HOH_DEG)
    h1 = ox + OH_BOHR * u
    h2 = ox + OH_BOHR * (math.cos(th) * u + math.sin(th) * v)
    pos = np.stack([ox, h1, h2], axis=1).reshape(-1, 3)
    elem = np.tile(np.array([O, H, H], dtype=np.int32), n_molecules)
    box = np.eye(3) * L
    return box, pos, elem


def noisy_frames(pos: np.ndarray, n_frames: int, sigma: float, seed: int,
                 box: np.ndarray | None = None, strain: float = 0.0):
    """Frames = base + N(0, sigma^2) per coordinate (+ isotropic strain in
    [-strain, strain], applied to positions and box).  Returns (boxes,
    frames) with shapes (F,3,3) and (F,N,3)."""
    rng = np.random.default_rng(seed)
    frames = np.empty((n_frames,) + pos.shape)
    boxes = np.empty((n_frames, 3, 3))
    for f in range(n_frames):
        s = 1.0 + (rng.uniform(-strain, strain) if strain > 0 else 0.0)
        frames[f] = pos * s + rng.normal(0.0, sigma, size=pos.shape)
        boxes[f] = (box if box is not None else np.eye(3)) * s
    return boxes, frames


def batch_structures(n_structures: int, seed: int, lo: int = 11,
                     hi: int = 171, device: str = "cpu"):
    """Independent water boxes with N ~ U[lo, hi] molecules each (density
    1.0 g/cm^3, O-O >= 4.7 bohr, seeded orientations), built by random
    sequential addition run for all structures at once with torch on
    `device`: every round proposes one oxygen per unfinished structure and
    accepts it if it keeps the minimum distance (minimum image) to the
    oxygens placed so far.  Returns a list of (box, positions, elements)."""
    import torch
    rng = np.random.default_rng(seed)
    counts = rng.integers(lo, hi + 1, size=n_structures)
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    S = n_structures
    nmax = int(counts.max())
    L = torch.tensor([box_length(int(c)) for c in counts],
                     dtype=torch.float64, device=dev)
    cnt = torch.tensor(counts, dtype=torch.int64, device=dev)
    placed = torch.zeros((S, nmax, 3), dtype=torch.float64, device=dev)
    npl = torch.zeros(S, dtype=torch.int64, device=dev)
    slot = torch.arange(nmax, device=dev)
    min2 = MIN_OO_BOHR ** 2
    rounds = 0
    while True:
        act = torch.nonzero(npl < cnt).flatten()
        if act.numel() == 0:
            break
        rounds += 1
        if rounds > 200000:
            raise RuntimeError("water placement did not converge")
        La = L[act]
        cand = torch.rand((act.numel(), 3), generator=g, dtype=torch.float64,
                          device=dev) * La[:, None]
        d = cand[:, None, :] - placed[act]
        d -= La[:, None, None] * torch.round(d / La[:, None, None])
        bad = ((d * d).sum(-1) < min2) & (slot[None, :] < npl[act, None])
        ok = ~bad.any(dim=1)
        acc = act[ok]
        placed[acc, npl[acc]] = cand[ok]
        npl[acc] += 1
    u = torch.randn((S, nmax, 3), generator=g, dtype=torch.float64,
                    device=dev)
    u /= torch.linalg.norm(u, dim=2, keepdim=True)
    v = torch.randn((S, nmax, 3), generator=g, dtype=torch.float64,
                    device=dev)
    v -= (v * u).sum(dim=2, keepdim=True) * u
    v /= torch.linalg.norm(v, dim=2, keepdim=True)
    th = math.radians(HOH_DEG)
    h1 = placed + OH_BOHR * u
    h2 = placed + OH_BOHR * (math.cos(th) * u + math.sin(th) * v)
    allpos = torch.stack([placed, h1, h2], dim=2).cpu().numpy()
    Ls = L.cpu().numpy()
    out = []
    for k in range(S):
        n = int(counts[k])
        pos = allpos[k, :n].reshape(-1, 3)
        elem = np.tile(np.array([O, H, H], dtype=np.int32), n)
        out.append((np.eye(3) * Ls[k], pos, elem))
    return out
