"""Host logic of the device trainer's driver (sdddst_b200/learned_train.py)
with a stand-in engine, no GPU: the step-size transient of every run is
skipped, every accepted step trains on J(h) and J(h/2), the Jacobian budget
is met exactly, and the file keeps the checkpoint with the lowest held-out
loss (the start included), not the last one."""
import json

import numpy as np

from sdddst_b200 import learned, learned_train


class FakeEngine:
    """Accepts every other step; the held-out loss of weights w is
    1 + (w[0] - 3)^2 until w[0] passes 5, then 100 (training overshoots);
    each applied training step adds 1 to w[0]."""

    def __init__(self, n, seed, log):
        self.n, self.seed, self.log = n, seed, log
        self.k = 0
        self.accepted = 0
        self.w = None

    def step(self):
        self.k += 1
        ok = self.k % 2 == 0
        self.accepted += ok
        return ok

    def scalars(self):
        return {"step_size": 1e-9 * (1 + self.accepted), "sim_time": 0.0, "energy": 0.0, "strain": 0.0}

    def config(self, which):
        return np.zeros((self.n, 3))

    def set_state(self, *a):
        pass

    def learned_train_init(self, w):
        self.w = np.array(w, dtype=np.float32, copy=True)

    def learned_train_step(self, h, probes=8, lr=0.0, seed=0, apply=True):
        x = float(self.w[0])
        loss = 1.0 + (x - 3.0) ** 2 if x <= 5.0 else 100.0
        if apply:
            self.log.append((self.n, self.seed, self.accepted, h))
            self.w[0] += 1.0
        return 50.0, loss

    def learned_train_weights(self):
        return self.w.copy()

    def close(self):
        pass


def test_driver_skips_transient_and_keeps_best_checkpoint(tmp_path, monkeypatch):
    log = []
    monkeypatch.setattr(learned_train, "_engine", lambda n, seed: FakeEngine(n, seed, log))
    w0 = np.zeros(learned.weight_count(), dtype=np.float32)
    monkeypatch.setattr(learned, "init_weights", lambda seed=0: w0.copy())
    out = tmp_path / "w.npz"
    learned_train.main(["--jacobians", "12", "--sizes", "4096", "8192", "--steps-per-run", "2", "--settle", "3",
                        "--heldout", "2", "--out", str(out)])
    # 2 accepted steps per run after 3 settling ones, 2 Jacobians each: 4 per run, 3 runs
    assert len(log) == 12
    assert all(acc > 3 for (_, _, acc, _) in log)
    assert [n for (n, _, _, _) in log] == [4096] * 4 + [8192] * 4 + [4096] * 4
    hs = [h for (_, _, _, h) in log]
    assert all(abs(hs[2 * k + 1] - 0.5 * hs[2 * k]) < 1e-24 for k in range(6))
    d = np.load(out)
    meta = json.loads(str(d["meta"]))
    # w[0] after the runs: 4, 8, 12 -> losses 2, 100, 100; the start (w[0] = 0) has 10
    assert meta["heldout_loss"]["B_plus_first_order"] == 10.0
    assert meta["heldout_loss"]["B_plus_learned_bf16"] == 2.0
    assert meta["heldout_loss"]["B_plus_last"] == 100.0
    assert meta["kept_checkpoint_after_jacobians"] == 4
    kept = (d["bf16"].astype(np.uint32) << 16).view(np.float32)
    assert kept[0] == 4.0
