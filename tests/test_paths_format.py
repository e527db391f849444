"""CPU: the .paths files this library writes are read by the reference's own BinReader
(include/IO/IOBinary.hpp:260-378, compiled in oracle/_ref).

qk_paths_write is the writer qk_run_config uses, on host arrays, so the format is
checked without a GPU: header (magic, version, element size, paths, steps, dt,
scale) and the row-major normalised payload, rescaled by the reader, at several
times of the grid, in the FP64 and the FP32 build of the reference."""
import ctypes as C

import numpy as np
import pytest


@pytest.mark.parametrize("precision,real_bytes", [(0, 8), (1, 4)])
def test_reference_binreader_reads_our_paths_file(tmp_path, ref, precision, real_bytes):
    from quantkos_b200 import _lib as L
    rng = np.random.default_rng(3)
    n_paths, n_steps, dt, scale = 37, 12, 0.25 / 12, 100.0
    S = scale * np.exp(np.cumsum(rng.normal(0.0, 0.02, (n_paths, n_steps)), axis=1))
    S = np.ascontiguousarray(S)
    path = tmp_path / "QuantKos.paths"
    st = L.lib().qk_paths_write(str(path).encode(), precision, n_paths, n_steps, dt, scale,
                                S.ctypes.data_as(C.POINTER(C.c_double)))
    assert st == L.QK_OK, L.lib().qk_last_error()
    stored = S / scale if precision == 0 else (S / scale).astype(np.float32).astype(np.float64)
    for j in (0, 5, n_steps - 1):
        got = ref.read_paths(str(tmp_path), path.name, (j + 1) * dt, n_paths, real_bytes)
        assert got.shape == (n_paths,)
        want = stored[:, j] * scale
        if precision == 0:
            np.testing.assert_allclose(got, want, rtol=1e-15)
        else:
            np.testing.assert_allclose(got, want, rtol=1e-6)
    with pytest.raises(RuntimeError, match="outside the simulated time grid"):
        ref.read_paths(str(tmp_path), path.name, (n_steps + 1) * dt, n_paths, real_bytes)
