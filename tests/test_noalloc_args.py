"""Matrix.spmv_noalloc checks its tensors on the host before anything reaches
the library: the allocation-free kernel has no bounds of its own, so a wrong
dtype, a non-contiguous or short tensor, or a tensor on another device must
raise here and never launch.  CPU only: the library is replaced by a stub
that fails the test if it is called."""
import types

import pytest


class _FakeCuda:
    """Stands in for a CUDA tensor (attributes the wrapper reads)."""

    def __init__(self, n, dtype, contiguous=True, device=0):
        import torch
        self.is_cuda = True
        self.dtype = dtype
        self._n = n
        self._contig = contiguous
        self.device = torch.device("cuda", device)

    def numel(self):
        return self._n

    def is_contiguous(self):
        return self._contig

    def data_ptr(self):
        return 0


@pytest.fixture
def stub_matrix(monkeypatch):
    import millefeuille as mf
    from millefeuille import _lib

    def never(*a, **k):
        raise AssertionError("mf_spmv_noalloc must not be called with rejected tensors")

    monkeypatch.setattr(_lib, "load", lambda: types.SimpleNamespace(mf_spmv_noalloc=never))

    class M(mf.Matrix):
        @property
        def info(self):
            return {"n_rows": 64, "n_cols": 80, "device": 0}

    return M(None)


def test_noalloc_rejects_bad_tensors_before_launch(stub_matrix):
    import torch
    f64, f32 = torch.float64, torch.float32
    good_x, good_y = _FakeCuda(80, f64), _FakeCuda(64, f64)
    cases = [
        (_FakeCuda(80, f32), good_y, TypeError),              # x not float64
        (good_x, _FakeCuda(64, f32), TypeError),              # y not float64
        (_FakeCuda(80, f64, contiguous=False), good_y, ValueError),
        (good_x, _FakeCuda(64, f64, contiguous=False), ValueError),
        (_FakeCuda(79, f64), good_y, ValueError),             # x shorter than n_cols
        (good_x, _FakeCuda(63, f64), ValueError),             # y shorter than n_rows
        (good_x, _FakeCuda(64, f64, device=1), ValueError),   # x and y on different devices
        (_FakeCuda(80, f64, device=1), _FakeCuda(64, f64, device=1), ValueError),   # not the matrix's device
    ]
    for x, y, exc in cases:
        with pytest.raises(exc):
            stub_matrix.spmv_noalloc(x, y)


def test_noalloc_rejects_host_tensors(stub_matrix):
    import torch
    with pytest.raises(TypeError):
        stub_matrix.spmv_noalloc(torch.zeros(80, dtype=torch.float64), torch.zeros(64, dtype=torch.float64))
