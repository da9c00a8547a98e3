"""The Arrow C data interface at the boundary (oxb_import_arrow /
oxb_export_arrow): a RecordBatch exported by pyarrow is read in place,
offsets and odd-bit validity offsets included, and a device batch comes
back as an Arrow struct array that pyarrow imports; both equal the plain
upload/download, bit for bit.  The buffers the reference's operator hands
its backend are these same Arrow buffers (columns.rs:192-289)."""
import numpy as np
import pyarrow as pa
import pytest

from compare import assert_batches_equal
from oxidelake_b200 import _abi
from oxidelake_b200.errors import Unsupported
from oxidelake_b200.params import Comparison as Cmp
from oxidelake_b200.params import Literal, compare

pytestmark = pytest.mark.gpu


def sample(n: int, seed: int = 5) -> pa.RecordBatch:
    rng = np.random.default_rng(seed)
    dim = 8
    return pa.RecordBatch.from_arrays(
        [
            pa.array(rng.integers(-1 << 40, 1 << 40, n), pa.int64(), mask=rng.random(n) < 0.1),
            pa.array(rng.standard_normal(n)),
            pa.array(rng.integers(-99, 99, n).astype(np.int32), mask=rng.random(n) < 0.2),
            pa.array(rng.standard_normal(n).astype(np.float32)),
            pa.FixedSizeListArray.from_arrays(pa.array(rng.standard_normal(n * dim).astype(np.float32)), dim,
                                              mask=pa.array(rng.random(n) < 0.05)),
        ],
        names=["k", "v", "q", "f", "emb"],
    )


@pytest.mark.parametrize("n", [0, 1, 1000, 3_000_001])
def test_round_trip_equals_the_plain_path(backend, stream, n):
    batch = sample(n)
    dev = backend.upload_arrow(stream, batch)
    assert dev.num_rows() == n
    assert_batches_equal(backend.download(stream, dev), batch)
    assert_batches_equal(backend.download_arrow(stream, dev), batch)
    plain = backend.upload(stream, batch)
    assert_batches_equal(backend.download_arrow(stream, plain), batch)


@pytest.mark.parametrize("start,length", [(13, 1000), (8, 4096), (1, 1), (777, 0)])
def test_sliced_batches_at_any_offset(backend, stream, start, length):
    """A slice carries its offset in the exported arrays: values start past
    it and a bitmap at an odd bit offset is re-based on the host."""
    whole = sample(6000, seed=9)
    part = whole.slice(start, length)
    dev = backend.upload_arrow(stream, part)
    assert_batches_equal(backend.download(stream, dev), part)


def test_unsupported_columns_are_refused_and_left_to_the_caller(backend, stream):
    batch = pa.RecordBatch.from_arrays([pa.array([1, 2, 3]), pa.array(["a", "b", "c"])], names=["k", "s"])
    backend.operator_stats(_abi.OP_TRANSFER, reset=True)
    with pytest.raises(Unsupported):
        backend.upload_arrow(stream, batch)
    assert backend.operator_stats(_abi.OP_TRANSFER)["unsupported"] == 1
    assert batch.column(1).to_pylist() == ["a", "b", "c"]  # still the caller's
    ok = backend.upload_arrow(stream, batch.select([0]))
    assert backend.download(stream, ok).column(0).to_pylist() == [1, 2, 3]


def test_export_of_a_device_result(backend, stream):
    """A filter's output (device memory the library allocated) leaves
    through the C data interface equal to the column-wise download."""
    batch = sample(200_000, seed=11)
    dev = backend.upload_arrow(stream, batch)
    out = backend.filter_project(stream, dev, compare(2, Cmp.Gt, Literal.int32(0)), [0, 4, 1])
    want = backend.download(stream, out)
    got = backend.download_arrow(stream, out)
    assert got.schema.names == ["k", "emb", "v"]
    assert_batches_equal(got, want)
    assert backend.last_call_stats()["bytes_d2h"] >= want.num_rows * (8 + 32 + 8)
