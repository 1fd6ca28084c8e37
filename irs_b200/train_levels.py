"""Train the level network of the adaptive IPM on labels the method generates.

For each training map (one star field per seed) the base lattice is shot, the
per-tile features computed, and a seeded sample of tiles labelled with the
smallest subdivision level whose interpolation stays within the tolerance of
the level-16 positions. The network is then trained on the device
(LevelNet.train) and saved with its feature standardisation.

  python -m irs_b200.train_levels --out irs_b200/data/level_net.npz

Defaults: the learned-adaptive configuration (Salpeter 0.08-1, kappa_tot 0.6,
shear 0.3, smooth fraction 0.3, 4096^2 map, half length 30) on seeds
2000-2063.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from .adaptive import AdaptiveIPM, LevelNet

CONFIG = dict(kappa_tot=0.6, shear=0.3, smooth_fraction=0.3, mass_function="salpeter", m_lower=0.08, m_upper=1.0,
              theta_star=1.0, half_length_y1=30.0, half_length_y2=30.0, num_pixels_y1=4096, num_pixels_y2=4096,
              write_histograms=0)


def label_maps(config, seeds, tiles_per_map, tolerance, sample_seed=0, verbose=True):
    """Features and labels of a seeded sample of tiles from one map per seed."""
    rng = np.random.default_rng(sample_seed)
    feats, labels = [], []
    for s in seeds:
        t0 = time.time()
        a = AdaptiveIPM(policy="uniform", level=1, audit_fraction=0.0, tolerance=tolerance,
                        **{**config, "random_seed": int(s)})
        a.run()
        f = a.features
        n = len(f)
        pick = np.sort(rng.choice(n, min(n, tiles_per_map), replace=False)).astype(np.int32)
        lab, _ = a.labels(pick)
        feats.append(f[pick])
        labels.append(lab)
        a.close()
        if verbose:
            print(f"seed {s}: {n} tiles, labelled {len(pick)}, classes {np.bincount(lab, minlength=5).tolist()}, "
                  f"{time.time() - t0:.1f} s", flush=True)
    return np.concatenate(feats), np.concatenate(labels)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="irs_b200/data/level_net.npz")
    ap.add_argument("--first-seed", type=int, default=2000)
    ap.add_argument("--maps", type=int, default=64)
    ap.add_argument("--tiles-per-map", type=int, default=2000)
    ap.add_argument("--tolerance", type=float, default=1e-4)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--num-pixels", type=int, default=4096)
    ap.add_argument("--half-length", type=float, default=30.0)
    a = ap.parse_args()
    cfg = {**CONFIG, "num_pixels_y1": a.num_pixels, "num_pixels_y2": a.num_pixels, "half_length_y1": a.half_length,
           "half_length_y2": a.half_length}
    seeds = range(a.first_seed, a.first_seed + a.maps)
    feat, lab = label_maps(cfg, seeds, a.tiles_per_map, a.tolerance)
    net, loss = LevelNet.train(feat, lab, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=0)
    acc = float(np.mean(net.predict(feat) == lab))
    print(f"trained on {len(lab)} tiles: loss {loss[0]:.3f} -> {loss[-1]:.3f}, accuracy {acc:.3f}, "
          f"classes {np.bincount(lab, minlength=5).tolist()}")
    net.save(a.out, tolerance=a.tolerance, seeds=np.array(list(seeds)), loss=loss, accuracy=acc,
             config=str(cfg), classes=np.bincount(lab, minlength=5))


if __name__ == "__main__":
    main()
