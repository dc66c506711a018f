"""Distillation of a small student atomic network from an n2p2 potential.

    python -m n2p2_b200.student train --teacher DIR --out DIR \
        [--frames 500] [--epochs 20] [--batch 4096] [--lr 1e-3] [--hidden 32]
        [--lr-final LR] [--decay-epochs 5] [--w-energy 1] [--w-force 1]
        [--sigma-max S] [--init STUDENT_DIR]

The teacher (an n2p2 potential directory) labels perturbed copies of a water
box with per-atom energies and forces in FP64.  The student -- one hidden
tanh layer of `hidden` neurons and a linear output per element, on the
teacher's own symmetry functions -- is trained on those labels with the
library's hand-written kernels (energy + force matching, Adam; see
n2p2b_student_train_step), using the FP32 symmetry functions of the mixed
form.  The result is a regular n2p2 potential directory (input.nn,
scaling.data, weights.%03zu.data) plus training_range.data, the per-SF range
of the training data that gates the student at inference
(Prediction.set_student_mode("gated")).
"""
from __future__ import annotations

import argparse
import os
import shutil
import time

import numpy as np

from . import synth

_SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co "
    "Ni Cu Zn Ga Ge As Se Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb "
    "Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb Lu Hf Ta W Re "
    "Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es "
    "Fm Md No Lr Rf Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og").split()

_NN_KEYS = ("global_hidden_layers_short", "global_nodes_short",
            "global_activation_short", "element_hidden_layers_short",
            "element_nodes_short", "element_activation_short",
            "normalize_nodes")


def atomic_number(symbol: str) -> int:
    return _SYMBOLS.index(symbol) + 1


def make_student_dir(teacher_dir: str, out_dir: str, num_sf: dict[str, int],
                     hidden: int = 16, seed: int = 0,
                     energy_bias: dict[str, float] | None = None):
    """Writes input.nn (the teacher's, with a 1-hidden-layer tanh network),
    the teacher's scaling.data and seeded initial weights (normal, variance
    1 / fan-in for standardized inputs: column l of W1 divided by sigma_l
    of scaling.data, floored at 1e-3 of the element's largest; output bias
    = the element's mean label energy).  Training then runs Adam on the
    standardized weights (per-input learning rate lr / sigma_l)."""
    os.makedirs(out_dir, exist_ok=True)
    lines = []
    with open(os.path.join(teacher_dir, "input.nn")) as fh:
        for ln in fh:
            w = ln.split()
            if w and w[0] in _NN_KEYS:
                continue
            lines.append(ln.rstrip("\n"))
    lines += ["", "# distilled student network",
              "global_hidden_layers_short 1",
              f"global_nodes_short {hidden}",
              "global_activation_short t l"]
    with open(os.path.join(out_dir, "input.nn"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    shutil.copyfile(os.path.join(teacher_dir, "scaling.data"),
                    os.path.join(out_dir, "scaling.data"))
    sigma = {}
    with open(os.path.join(teacher_dir, "scaling.data")) as fh:
        for ln in fh:
            w = ln.split()
            if len(w) < 6 or w[0].startswith("#"):
                continue
            sigma.setdefault(int(w[0]), {})[int(w[1])] = float(w[5])
    syms = sorted(num_sf, key=atomic_number)
    rng = np.random.default_rng(seed)
    for sym, nin in num_sf.items():
        W1 = rng.normal(0.0, 1.0 / np.sqrt(nin), (hidden, nin))
        sg = sigma.get(syms.index(sym) + 1, {})
        if sg:
            sv = np.array([sg.get(l + 1, 1.0) for l in range(nin)])
            W1 /= np.maximum(sv, 1e-3 * sv.max())[None, :]
        b1 = np.zeros(hidden)
        w2 = rng.normal(0.0, 1.0 / np.sqrt(hidden), hidden)
        b2 = (energy_bias or {}).get(sym, 0.0)
        vals = []
        # NeuralNetwork::setConnections order: per layer, for each input j,
        # for each neuron k: W[k][j]; then the layer's biases.
        for j in range(nin):
            vals.extend(W1[:, j])
        vals.extend(b1)
        vals.extend(w2)
        vals.append(b2)
        path = os.path.join(out_dir,
                            "weights.%03d.data" % atomic_number(sym))
        with open(path, "w") as fh:
            fh.write(f"# initial student weights of element {sym}\n")
            fh.writelines(f"{v:24.16E}\n" for v in vals)


def training_frames(n_frames: int = 500, sigma: float = 0.15,
                    strain: float = 0.03, n_mol: int = 8192,
                    base_seed: int = 2026, seed: int = 7,
                    sigma_max: float | None = None):
    """Perturbed copies of one water box: Gaussian position noise `sigma`
    (with `sigma_max`, a width drawn per frame from U[sigma, sigma_max]) and
    a random isotropic strain in [-strain, strain] per frame."""
    box, pos, elem = synth.water_box(n_mol, base_seed)
    rng = np.random.default_rng(seed)
    frames = []
    for _ in range(n_frames):
        s = 1.0 + rng.uniform(-strain, strain)
        sig = sigma if sigma_max is None else rng.uniform(sigma, sigma_max)
        x = pos * s + rng.normal(0.0, sig, pos.shape)
        frames.append((box * s, x))
    return frames, elem


def label_frames(teacher_dir: str, frames, elem, device: int = 0):
    """FP64 teacher atomic energies [F, n] and forces [F, n, 3] on the GPU."""
    import torch
    from .mode import Prediction
    t = Prediction(teacher_dir, device=device)
    t.setup()
    t.setup_symmetry_function_statistics(False, False, False, False)
    E, Fo = [], []
    for box, x in frames:
        t.set_structure(x, elem, box)
        t.evaluate_nnp(True)
        E.append(torch.tensor(t.atomic_energies(), dtype=torch.float64))
        Fo.append(torch.tensor(t.forces(), dtype=torch.float64))
    t.close()
    dev = torch.device("cuda", device)
    return torch.stack(E).to(dev), torch.stack(Fo).to(dev)


def train(teacher_dir: str, student_dir: str, frames, elem, labels,
          epochs: int = 20, batch: int = 4096, lr: float = 1e-3,
          w_energy: float = 1.0, w_force: float = 1.0, seed: int = 11,
          device: int = 0, log=print, lr_final: float | None = None,
          decay_epochs: int = 5):
    """Trains the student in `student_dir` in place and writes it back.
    With `lr_final`, the learning rate stays `lr` and then falls linearly
    to `lr_final` over the last `decay_epochs` epochs."""
    import torch
    from .mode import Prediction
    E, Fo = labels
    p = Prediction(teacher_dir, device=device)
    p.setup()
    p.setup_symmetry_function_statistics(False, False, False, False)
    p.set_precision("mixed")
    p.setup_student(student_dir)
    n = len(elem)
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", device)
    t0 = time.perf_counter()
    steps = 0
    p.student_update_range(reset=True)
    history = []
    for ep in range(epochs):
        lr_ep = lr
        if lr_final is not None and ep >= epochs - decay_epochs:
            f = (ep - (epochs - decay_epochs) + 1) / decay_epochs
            lr_ep = lr + (lr_final - lr) * f
        order = rng.permutation(len(frames))
        le = lf = 0.0
        cnt = 0
        for fi in order:
            box, x = frames[fi]
            p.set_structure(x, elem, box)
            p.calculate_neighbor_list()
            p.calculate_symmetry_function_groups(True)
            if ep == 0:
                p.student_update_range()
            perm = torch.tensor(rng.permutation(n).astype(np.int32),
                                device=dev)
            for b0 in range(0, n, batch):
                idx = perm[b0:b0 + batch].contiguous()
                want = b0 + batch >= n
                r = p.student_train_step(E[fi], Fo[fi], idx, w_energy,
                                         w_force, lr_ep, want_loss=want)
                steps += 1
                if r is not None:
                    le += r[0]
                    lf += r[1]
                    cnt += 1
        history.append((le / max(cnt, 1), lf / max(cnt, 1)))
        log(f"epoch {ep + 1}/{epochs}: energy loss {history[-1][0]:.3e} "
            f"force loss {history[-1][1]:.3e} ({steps} steps, "
            f"{time.perf_counter() - t0:.0f} s)")
    p.student_write(student_dir)
    p.close()
    return {"steps": steps, "seconds": time.perf_counter() - t0,
            "history": history}


def distill(teacher_dir: str, out_dir: str, n_frames=500, epochs=20,
            batch=4096, lr=1e-3, hidden=32, seed=0, device=0, log=print,
            lr_final=None, w_energy=1.0, w_force=1.0, decay_epochs=5,
            init=None, sigma=0.15, sigma_max=None):
    """Labels the training frames with the teacher and trains a student in
    `out_dir`: a fresh one, or with `init` a copy of that student directory
    (its network and weights) trained further."""
    from .mode import Prediction
    frames, elem = training_frames(n_frames, sigma=sigma, sigma_max=sigma_max)
    log(f"labelling {len(frames)} frames with the FP64 teacher")
    labels = label_frames(teacher_dir, frames, elem, device)
    host = Prediction(teacher_dir, device=-1)
    host.setup()
    syms = host.elements
    num_sf = {s: host.num_symmetry_functions(e) for e, s in enumerate(syms)}
    Ecpu = labels[0][0].cpu().numpy()
    bias = {s: float(Ecpu[elem == e].mean()) for e, s in enumerate(syms)}
    host.close()
    if init is None:
        make_student_dir(teacher_dir, out_dir, num_sf, hidden, seed, bias)
    else:
        os.makedirs(out_dir, exist_ok=True)
        for f in os.listdir(init):
            if f != "training.log" and os.path.isfile(os.path.join(init, f)):
                shutil.copyfile(os.path.join(init, f),
                                os.path.join(out_dir, f))
    return train(teacher_dir, out_dir, frames, elem, labels, epochs, batch,
                 lr, w_energy, w_force, device=device, log=log,
                 lr_final=lr_final, decay_epochs=decay_epochs)


def main():
    a = argparse.ArgumentParser()
    sub = a.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--teacher", required=True)
    t.add_argument("--out", required=True)
    t.add_argument("--frames", type=int, default=500)
    t.add_argument("--epochs", type=int, default=20)
    t.add_argument("--batch", type=int, default=4096)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--hidden", type=int, default=32)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--lr-final", type=float, default=None,
                   help="decay the learning rate linearly to this value "
                        "over the last --decay-epochs epochs")
    t.add_argument("--decay-epochs", type=int, default=5)
    t.add_argument("--w-energy", type=float, default=1.0)
    t.add_argument("--w-force", type=float, default=1.0)
    t.add_argument("--sigma", type=float, default=0.15,
                   help="position noise of the training frames (bohr)")
    t.add_argument("--sigma-max", type=float, default=None,
                   help="draw the noise per frame from U[sigma, sigma-max]")
    t.add_argument("--init", default=None,
                   help="continue training this student directory")
    args = a.parse_args()
    r = distill(args.teacher, args.out, args.frames, args.epochs, args.batch,
                args.lr, args.hidden, args.seed, lr_final=args.lr_final,
                w_energy=args.w_energy, w_force=args.w_force,
                decay_epochs=args.decay_epochs, init=args.init,
                sigma=args.sigma, sigma_max=args.sigma_max)
    print(f"trained: {r['steps']} steps in {r['seconds']:.0f} s")


if __name__ == "__main__":
    main()
