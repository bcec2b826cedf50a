"""The learned LOD surrogate: weight files, the fit, training pairs from the plain solver, and the
judge's calibration.

The operator, its training step and its judge run in the library (gell_surrogate_train_pair,
gell_lod_surrogate: hand-written tcgen05 kernels); this module drives the fit and the
calibration.  Training pairs come from the plain LOD solver (the reference's LODsolver,
include/LODkernel.cuh:280-300, bit-exact in this library): input (p, uptake map, shell) -> p
after `substeps` substeps, over seeded jittered-lattice
spheroids with the large plain-method workload's statistics (volume fraction 0.6, radii N(5, 0.5)
um) placed at random centres with seeded Ki-67 states.  The surrogate stands in for the substeps of
a quasi-steady field between mechanics steps, so each spheroid's field is first relaxed from the
boundary value by a few hundred plain substeps, and each pair is one block of the running model:
a few mechanics steps (FM_update) move the cells, PreLOD rebuilds the uptake map, and the field
before and after `substeps` plain substeps form the pair.

Weight file: 8-byte magic b"GSUR0002", int32 substeps, float32 rate_scale, float32 threshold,
int32 input_kind (GELL_OPT_SURROGATE_INPUT: 0 the field, 1 the change of one plain substep),
int64 count, then `count` float32 weights in gell_surrogate_load's order (little-endian).  Files
with the magic b"GSUR0001" have no input_kind (the field form).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

MAGIC = b"GSUR0002"
MAGIC_V1 = b"GSUR0001"
# weights fitted for oxygen (the large workload's parameters) on 256^3 grids of 10 um
DEFAULT_WEIGHTS = __import__("os").path.join(__import__("os").path.dirname(__file__), "data", "o2_surrogate_256.gsur")
SHAPES = [(3, 32)] + [(32, 32)] * 8 + [(32, 1)]  # (cin, cout) of the ten convolutions


@dataclass
class SurrogateWeights:
    weights: np.ndarray
    substeps: int = 50
    rate_scale: float = 0.1
    threshold: float = 1e-3
    input_kind: int = 0


def save_weights(path: str, sw: SurrogateWeights) -> None:
    w = np.ascontiguousarray(sw.weights, np.float32).reshape(-1)
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<iffiq", sw.substeps, sw.rate_scale, sw.threshold, sw.input_kind, w.size))
        f.write(w.astype("<f4").tobytes())


def load_weights(path: str) -> SurrogateWeights:
    with open(path, "rb") as f:
        magic = f.read(8)
        if magic == MAGIC:
            substeps, rate_scale, threshold, input_kind, n = struct.unpack("<iffiq", f.read(24))
        elif magic == MAGIC_V1:
            substeps, rate_scale, threshold, n = struct.unpack("<iffq", f.read(20))
            input_kind = 0
        else:
            raise ValueError(f"{path}: not a surrogate weight file")
        w = np.frombuffer(f.read(4 * n), "<f4").astype(np.float32)
    if w.size != n:
        raise ValueError(f"{path}: truncated")
    return SurrogateWeights(w, substeps, rate_scale, threshold, input_kind)


def weight_count() -> int:
    return sum(co * ci * 27 + co for ci, co in SHAPES)


def shell_mask(N: int) -> np.ndarray:
    """The four boundary layers of every face (Setboundary, include/LODkernel.cuh:112-136)."""
    g = np.arange(N)
    s = (g < 2) | (g > N - 3)
    return (s[:, None, None] | s[None, :, None] | s[None, None, :]).ravel()


def init_weights(seed: int = 11) -> np.ndarray:
    """Initial weights: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for every layer but the last, which is
    zero, so the fit starts from the identity map q = p."""
    rng = np.random.Generator(np.random.Philox(seed))
    parts = []
    for l, (ci, co) in enumerate(SHAPES):
        if l == len(SHAPES) - 1:
            parts += [np.zeros(co * ci * 27, np.float32), np.zeros(co, np.float32)]
        else:
            bound = 1.0 / np.sqrt(ci * 27)
            parts += [rng.uniform(-bound, bound, co * ci * 27).astype(np.float32),
                      rng.uniform(-bound, bound, co).astype(np.float32)]
    return np.concatenate(parts)


def seed_spheroid(sim, rng, N: int, cells: tuple[int, int], length: float, warm: tuple[int, int]) -> None:
    """A new seeded spheroid in `sim` (cell count log-uniform in `cells`, random centre), its field
    relaxed from the boundary value by a number of plain substeps drawn from `warm`."""
    import gell_b200 as gb
    L = N * length
    n = int(np.exp(rng.uniform(np.log(cells[0]), np.log(cells[1]))))
    a = (4.0 / 3.0 * np.pi * 125.0 / 0.6) ** (1.0 / 3.0)
    r = a * (3.0 * n / (4.0 * np.pi)) ** (1.0 / 3.0)
    lo, hi = r + 4 * length, L - r - 4 * length
    centre = rng.uniform(lo, hi, 3) if hi > lo else np.full(3, L / 2)
    c = gb.lattice_spheroid(n, centre, int(rng.integers(1 << 30)), length, N)
    c = gb.seed_ki67_states(c, int(rng.integers(1 << 30)))
    sim.import_cells(c)
    sim.set_field(0, np.full(N ** 3, sim_boundary(gb), np.float32))
    sim.PreLOD()
    sim.LODsolver(int(rng.integers(warm[0], warm[1] + 1)), 0)


class PairSource:
    """Training or validation pairs from a few contexts, each following one spheroid for `blocks`
    blocks before the next spheroid replaces it.  A new spheroid's field is relaxed by a number of
    plain substeps drawn from `warm`; every block moves the cells by a number of mechanics steps
    drawn from `moves`."""

    def __init__(self, N: int, cells: tuple[int, int], seed: int, substeps: int = 50, blocks: int = 8,
                 contexts: int = 4, length: float = 10.0, warm: tuple[int, int] = (300, 1000),
                 moves: tuple[int, int] = (1, 5)):
        import gell_b200 as gb
        self.gb, self.N, self.cells, self.substeps, self.blocks, self.length = gb, N, cells, substeps, blocks, length
        self.warm, self.moves = warm, moves
        self.rng = np.random.Generator(np.random.Philox(seed))
        self.sims = []
        self.left = []
        for _ in range(contexts):
            sim = gb.Simulation(voxel_num=N, voxel_length=length, max_cell_num=cells[1])
            sim.add_substrate(gb.oxygen())
            self.sims.append(sim)
            self.left.append(0)
        self.k = 0

    def _reseed(self, sim) -> None:
        seed_spheroid(sim, self.rng, self.N, self.cells, self.length, self.warm)

    def next(self):
        """(p, rate, target) as float32 arrays of N^3 values."""
        i = self.k % len(self.sims)
        self.k += 1
        sim = self.sims[i]
        if self.left[i] == 0:
            self._reseed(sim)
            self.left[i] = self.blocks
        for _ in range(int(self.rng.integers(self.moves[0], self.moves[1] + 1))):
            sim.FM_update()
        sim.PreLOD()
        p = sim.field(0)
        rate = sim.dump_rate(0)
        sim.LODsolver(self.substeps, 0)
        self.left[i] -= 1
        return p, rate, sim.field(0)

    def close(self) -> None:
        for s in self.sims:
            s.close()


def sim_boundary(gb) -> float:
    return float(gb.oxygen().boundary)


def train(N: int = 256, pairs: int = 2000, substeps: int = 50, rate_scale: float = 0.1, seed: int = 11,
          cells: tuple[int, int] = (150_000, 450_000), lr: float = 3e-4, max_seconds: float = float("inf"),
          blocks: int = 4, warm: tuple[int, int] = (300, 1000), moves: tuple[int, int] = (1, 5),
          input_kind: int = 0, log=print) -> SurrogateWeights:
    """Fit the operator with the library's training kernels (gell_surrogate_train_pair): one pair per
    step, never reused, from one context that follows a seeded spheroid for `blocks` blocks (each
    block: 1-5 mechanics steps, PreLOD, the pair) before the next spheroid replaces it.  Adam with
    the gradient clipped to norm 1 and the rate on a cosine from `lr` to 0; the loss is the mean
    squared error inside the shell in units of the boundary value (input_kind 0) or of the largest
    one-substep change (input_kind 1, GELL_OPT_SURROGATE_INPUT).  Stops after `max_seconds`."""
    import math
    import time

    import gell_b200 as gb

    rng = np.random.Generator(np.random.Philox(seed))
    t0 = time.time()
    done = 0
    with gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=cells[1]) as sim:
        sim.add_substrate(gb.oxygen())
        sim.surrogate_train_init(0, init_weights(seed), substeps, rate_scale, input_kind)
        left = 0
        for it in range(pairs):
            if left == 0:
                seed_spheroid(sim, rng, N, cells, 10.0, warm)
                left = blocks
            for _ in range(int(rng.integers(moves[0], moves[1] + 1))):
                sim.FM_update()
            sim.PreLOD()
            rate = 0.5 * lr * (1.0 + math.cos(math.pi * it / pairs))
            report = it % 50 == 0 or it == pairs - 1
            loss = sim.surrogate_train_pair(0, rate, want_loss=report)
            left -= 1
            done = it + 1
            if report:
                log(f"pair {it} ({time.time() - t0:.0f} s): rmse {math.sqrt(loss):.3e}")
            if time.time() - t0 > max_seconds:
                log(f"stopped after {done} pairs ({max_seconds:.0f} s)")
                break
        w = sim.surrogate_train_read(0, 0)
    log(f"fit: {done} pairs in {time.time() - t0:.1f} s")
    return SurrogateWeights(w, substeps, rate_scale, 0.0, input_kind)


def calibrate(sw: SurrogateWeights, N: int = 256, pairs: int = 64, seed: int = 1234,
              cells: tuple[int, int] = (150_000, 450_000), tol: float = 0.01, log=print,
              warm: tuple[int, int] = (300, 1000), moves: tuple[int, int] = (1, 5), margin: float = 1.0):
    """Run the library's operator and judge on held-out pairs and set the threshold: the judge's
    residual r bounds the error e (L-infinity inside the shell, units of the boundary value) on
    these pairs as e <= kappa * r with kappa the largest ratio seen; threshold = tol / (kappa *
    margin).  `warm` and `moves` choose the pairs' regime (see PairSource): fields relaxed for
    800-1500 substeps with one mechanics step per block are the quasi-steady fields the surrogate
    stands in for.  Returns (threshold, [(r, e)])."""
    import gell_b200 as gb

    src = PairSource(N, cells, seed, sw.substeps, warm=warm, moves=moves)
    b = sim_boundary(gb)
    inner = ~shell_mask(N)
    out = []
    try:
        with gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=cells[1]) as sim:
            sim.add_substrate(gb.oxygen())
            sim.surrogate_load(0, sw.weights, sw.substeps, sw.rate_scale, 1e30, sw.input_kind)
            for _ in range(pairs):
                i = src.k % len(src.sims)
                p, rate, tgt = src.next()
                # the same state in the judging context: cells of the source context
                sim.import_cells(src.sims[i].export_cells())
                sim.PreLOD()
                sim.set_field(0, p)
                _, r = sim.lod_surrogate(0)
                q = sim.field(0)
                e = float(np.abs(q - tgt)[inner].max() / b)
                out.append((r, e))
                log(f"  r {r:.3e}  e {e:.3e}  identity {float(np.abs(p - tgt)[inner].max() / b):.3e}")
    finally:
        src.close()
    kappa = max(e / max(r, 1e-12) for r, e in out)
    thr = tol / (kappa * margin)
    log(f"calibration: kappa {kappa:.3g}, threshold {thr:.3e}, accepted {sum(r <= thr for r, _ in out)}/{len(out)}")
    return thr, out


def time_inference(N: int = 128, reps: int = 3, ring: bool = True, path: str | None = None, cells: int = 40_000,
                   log=print) -> dict:
    """Per-kernel device times of `reps` inferences of the operator on an N^3 grid holding a
    quasi-steady spheroid of `cells` cells (CUDA events per launch, the library's profiler)."""
    import gell_b200 as gb

    sw = load_weights(path or DEFAULT_WEIGHTS)
    c = gb.lattice_spheroid(cells, N * 10.0 / 2, 5, 10.0, N)
    with gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=cells) as sim:
        sim.add_substrate(gb.oxygen())
        sim.import_cells(c)
        sim.PreLOD()
        sim.LODsolver(100, 0)
        sim.set_conv_ring(ring)
        sim.surrogate_load(0, sw.weights, sw.substeps, sw.rate_scale, sw.threshold, sw.input_kind)
        sim.surrogate_infer(0)  # first launches (module loading) outside the timing
        sim.profile(True)
        sim.profile_read(reset=True)
        for _ in range(reps):
            sim.surrogate_infer(0)
        prof = sim.profile_read(reset=True)
    out = {k: {"launches": v[0] / reps, "ms_per_inference": v[1] / reps, "ms_per_launch": v[1] / v[0]}
           for k, v in prof.items()}
    log(out)
    return out


def time_training(N: int = 128, reps: int = 2, cells: int = 40_000, log=print) -> dict:
    """Per-kernel device times of `reps` training pairs (gell_surrogate_train_pair) on an N^3 grid
    holding a quasi-steady spheroid of `cells` cells, starting from the packaged weights."""
    import gell_b200 as gb

    sw = load_weights(DEFAULT_WEIGHTS)
    c = gb.lattice_spheroid(cells, N * 10.0 / 2, 5, 10.0, N)
    with gb.Simulation(voxel_num=N, voxel_length=10.0, max_cell_num=cells) as sim:
        sim.add_substrate(gb.oxygen())
        sim.import_cells(c)
        sim.PreLOD()
        sim.LODsolver(100, 0)
        sim.surrogate_train_init(0, sw.weights, sw.substeps, sw.rate_scale, sw.input_kind)
        sim.surrogate_train_pair(0, 1e-5)  # first launches (module loading) outside the timing
        sim.profile(True)
        sim.profile_read(reset=True)
        for _ in range(reps):
            sim.surrogate_train_pair(0, 1e-5, want_loss=False)
        prof = sim.profile_read(reset=True)
    out = {k: {"launches": v[0] / reps, "ms_per_pair": v[1] / reps} for k, v in prof.items()}
    log(out)
    return out


def main(argv=None) -> int:
    import argparse
    import sys
    import time

    argv = sys.argv[1:] if argv is None else argv
    if argv and argv[0] == "time":
        tp = argparse.ArgumentParser(description="Time the operator's kernels on an N^3 grid.")
        tp.add_argument("--N", type=int, default=128)
        tp.add_argument("--reps", type=int, default=3)
        tp.add_argument("--no-ring", action="store_true")
        tp.add_argument("--weights", default=None)
        t = tp.parse_args(argv[1:])
        time_inference(t.N, t.reps, not t.no_ring, t.weights)
        return 0
    if argv and argv[0] == "time-train":
        tp = argparse.ArgumentParser(description="Time the training kernels on an N^3 grid.")
        tp.add_argument("--N", type=int, default=128)
        tp.add_argument("--reps", type=int, default=2)
        t = tp.parse_args(argv[1:])
        time_training(t.N, t.reps)
        return 0
    if argv and argv[0] == "calibrate":
        cp = argparse.ArgumentParser(description="Recalibrate the judge of a weight file on held-out pairs "
                                                 "(`... calibrate --weights IN --out OUT`).")
        cp.add_argument("--weights", default=DEFAULT_WEIGHTS)
        cp.add_argument("--out", required=True)
        cp.add_argument("--N", type=int, default=256)
        cp.add_argument("--pairs", type=int, default=64)
        cp.add_argument("--seed", type=int, default=4321)
        cp.add_argument("--warm", type=int, nargs=2, default=(800, 1500))
        cp.add_argument("--moves", type=int, nargs=2, default=(1, 1))
        cp.add_argument("--cells", type=int, nargs=2, default=(150_000, 450_000))
        cp.add_argument("--margin", type=float, default=1.1)
        cp.add_argument("--tol", type=float, default=0.01)
        c = cp.parse_args(argv[1:])
        sw = load_weights(c.weights)
        t1 = time.time()
        sw.threshold, pts = calibrate(sw, c.N, c.pairs, c.seed, tuple(c.cells), c.tol,
                                      log=lambda m: print(m, flush=True), warm=tuple(c.warm), moves=tuple(c.moves),
                                      margin=c.margin)
        print(f"calibration: {c.pairs} pairs in {time.time() - t1:.1f} s", flush=True)
        save_weights(c.out, sw)
        return 0
    if argv and argv[0] == "fit":
        argv = argv[1:]
    ap = argparse.ArgumentParser(description="Fit the LOD surrogate of oxygen and calibrate its judge "
                                             "(`python -m gell_b200.surrogate [fit] --out FILE`; "
                                             "`... time --N 128` times the operator's kernels, "
                                             "`... time-train --N 128` those of a training pair).")
    ap.add_argument("--out", required=True)
    ap.add_argument("--N", type=int, default=256)
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--val-pairs", type=int, default=64)
    ap.add_argument("--substeps", type=int, default=50)
    ap.add_argument("--lr", type=float, default=3e-4)
    ap.add_argument("--tol", type=float, default=0.01)
    ap.add_argument("--max-seconds", type=float, default=float("inf"))
    ap.add_argument("--input", choices=("field", "delta"), default="field",
                    help="the operator's input: the field p / b, or the change of one plain substep")
    ap.add_argument("--margin", type=float, default=1.1, help="calibration safety margin")
    a = ap.parse_args(argv)
    sw = train(a.N, a.pairs, a.substeps, lr=a.lr, max_seconds=a.max_seconds, input_kind=int(a.input == "delta"),
               log=lambda m: print(m, flush=True))
    t1 = time.time()
    # the judge is calibrated on the regime the surrogate stands in for: quasi-steady fields
    sw.threshold, pts = calibrate(sw, a.N, a.val_pairs, tol=a.tol, log=lambda m: print(m, flush=True),
                                  warm=(800, 1500), moves=(1, 1), margin=a.margin)
    print(f"calibration: {a.val_pairs} pairs in {time.time() - t1:.1f} s", flush=True)
    save_weights(a.out, sw)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
