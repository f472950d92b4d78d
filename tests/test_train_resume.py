"""Resuming the preconditioner training from a checkpoint (CPU, the network
mocked): a run interrupted after a checkpoint and resumed from it takes the
same batch draws and learning rates as the uninterrupted run, and a resume
with other settings than the checkpoint's is refused."""
import numpy as np
import pytest
import torch

from similie_b200.precond import write_checkpoint
from similie_b200.train_precond import check_resume, train


class _Stop(Exception):
    pass


class _MockNet:
    """Records every train_step (grid size, the drawn pairs' ids, lr); raises
    after `stop_after` steps to emulate a killed run."""

    def __init__(self, stop_after=None):
        self.calls = []
        self.stop_after = stop_after

    def train_step(self, shapes, nu, b, x, lr):
        if self.stop_after is not None and len(self.calls) == self.stop_after:
            raise _Stop()
        n = shapes[0][0]
        self.calls.append((n, tuple(b.view(len(shapes), -1)[:, 0].tolist()), lr))
        return 1.0

    def save_checkpoint(self, path, step, seed, extra=None):
        write_checkpoint(path, np.zeros(4, dtype=np.float32), step, seed, extra)


def _pairs():
    out = {}
    for n, count in ((4, 5), (6, 3), (8, 7)):
        out[n] = [(torch.ones(n * n), torch.full((n * n,), float(100 * n + i)), torch.zeros(n * n))
                  for i in range(count)]
    return out


def test_resumed_run_repeats_the_uninterrupted_draws_and_schedule(tmp_path):
    pairs = _pairs()
    steps, batch, lr, seed = 12, 3, 1e-3, 5
    full = _MockNet()
    train(full, pairs, steps, batch, lr, seed)
    ck = tmp_path / "ck.bin"
    first = _MockNet(stop_after=7)
    with pytest.raises(_Stop):
        train(first, pairs, steps, batch, lr, seed, checkpoint=str(ck), checkpoint_every=4)
    start = check_resume(str(ck), seed, steps, batch, lr)
    assert start == 4
    rest = _MockNet()
    train(rest, pairs, steps, batch, lr, seed, start=start)
    assert first.calls[:start] + rest.calls == full.calls
    assert not (tmp_path / "ck.bin.tmp").exists()


@pytest.mark.parametrize("field,value", [("seed", 6), ("steps", 13), ("batch", 4), ("lr", 2e-3)])
def test_resume_with_other_settings_is_refused(tmp_path, field, value):
    ck = tmp_path / "ck.bin"
    write_checkpoint(str(ck), np.zeros(4, dtype=np.float32), 4, 5, {"steps": 12, "batch": 3, "lr": 1e-3})
    settings = {"seed": 5, "steps": 12, "batch": 3, "lr": 1e-3}
    settings[field] = value
    with pytest.raises(ValueError, match=field):
        check_resume(str(ck), **settings)
