"""Native handles collected during a CUDA graph capture are destroyed after
it: destroying frees device memory, which would end the capture with an
error (host logic only; the capture state is faked)."""
import torch

from dgfs1d_gpu_b200 import _native as nat


def test_release_defers_destruction_during_a_capture(monkeypatch):
    freed = []
    monkeypatch.setattr(torch.cuda, 'is_available', lambda: True)
    monkeypatch.setattr(torch.cuda, 'is_current_stream_capturing', lambda: True)
    nat.release(freed.append, 'a')
    nat.release(freed.append, 'b')
    assert freed == []
    monkeypatch.setattr(torch.cuda, 'is_current_stream_capturing', lambda: False)
    nat.release(freed.append, 'c')
    assert sorted(freed) == ['a', 'b', 'c'] and freed[-1] == 'c'
    assert nat._deferred == []
