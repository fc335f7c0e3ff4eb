"""The native GIFTI payload decoder (``csg_gifti_decode``) against Python's base64 and zlib.

Host-only: the decoder touches no device.  Every case decodes to exactly the bytes
``base64.b64decode`` / ``zlib.decompress`` give, or fails with ``ValueError`` where they
fail (or where the payload disagrees with the array size in its header).
"""

from __future__ import annotations

import base64
import zlib

import numpy as np
import pytest


def _decode(text: bytes, gzip: bool, size: int, lengths=None) -> tuple[bytes, int]:
    from cat_surface_gpu_b200 import gifti

    out = np.empty(size, dtype=np.uint8)
    check = gifti._decode_payload(text, gzip, lengths, out)
    return out.tobytes(), check


@pytest.mark.parametrize("size", [0, 1, 2, 3, 4, 5, 47, 48, 49, 4096, 65537, 300_001])
def test_base64_matches_python_at_every_padding(native_library, size):
    raw = np.random.default_rng(size).bytes(size)
    text = base64.b64encode(raw)
    got, check = _decode(text, False, size)
    assert got == raw
    assert check == zlib.adler32(raw)


def test_whitespace_anywhere_is_skipped(native_library):
    raw = np.random.default_rng(1).bytes(10_000)
    text = base64.b64encode(raw).decode()
    wrapped = "\n  " + "\r\n\t".join(text[i:i + 61] for i in range(0, len(text), 61)) + " \n"
    spaced = " ".join(text)  # a space between every character, padding included
    for variant in (wrapped, spaced):
        assert _decode(variant.encode(), False, len(raw))[0] == raw


@pytest.mark.parametrize("bad", [
    b"QUJD!A==",      # a character outside the alphabet
    b"QUJDRA=A",      # data after padding
    b"QUJDR===",      # padding too early
    b"QUJDRA",        # an incomplete group
    b"QUJDRA==QUJD",  # data after a padded group
])
def test_malformed_base64_is_refused(native_library, bad):
    with pytest.raises(ValueError):
        _decode(bad, False, 4)


def test_size_must_match_the_header(native_library):
    raw = bytes(range(30))
    text = base64.b64encode(raw)
    with pytest.raises(ValueError, match="longer"):
        _decode(text, False, 29)
    with pytest.raises(ValueError, match="holds"):
        _decode(text, False, 31)
    z = base64.b64encode(zlib.compress(raw))
    assert _decode(z, True, 30)[0] == raw
    with pytest.raises(ValueError, match="more than"):
        _decode(z, True, 29)
    with pytest.raises(ValueError, match="holds"):
        _decode(z, True, 31)


@pytest.mark.parametrize("level", [0, 1, 6, 9])
def test_zlib_stream_matches_python(native_library, level):
    rng = np.random.default_rng(level)
    raw = (rng.integers(0, 50, size=200_000, dtype=np.int32)).tobytes()
    z = zlib.compress(raw, level)
    got, check = _decode(base64.b64encode(z), True, len(raw))
    assert got == zlib.decompress(z)
    assert check == zlib.adler32(raw) == int.from_bytes(z[-4:], "big")
    # trailing bytes after the stream are ignored, as zlib.decompress ignores them
    assert _decode(base64.b64encode(z + b"tail"), True, len(raw))[0] == raw


def test_corrupt_and_truncated_streams_are_refused(native_library):
    raw = np.arange(50_000, dtype=np.int32).tobytes()
    z = bytearray(zlib.compress(raw, 6))
    with pytest.raises(ValueError, match="zlib"):
        _decode(base64.b64encode(bytes(z[: len(z) // 2])), True, len(raw))
    flipped = bytearray(z)
    flipped[-1] ^= 0x01  # the Adler-32 check
    with pytest.raises(ValueError, match="check"):
        _decode(base64.b64encode(bytes(flipped)), True, len(raw))
    garbage = bytearray(z)
    garbage[len(z) // 2: len(z) // 2 + 8] = b"\xff" * 8
    with pytest.raises(ValueError):
        _decode(base64.b64encode(bytes(garbage)), True, len(raw))
    with pytest.raises(ValueError):
        _decode(base64.b64encode(b"\x78\x01"), True, len(raw))


def test_chunked_stream_inflates_in_parallel_and_checks_each_chunk(native_library):
    from cat_surface_gpu_b200 import gifti

    raw = np.random.default_rng(3).integers(0, 200, size=900_000, dtype=np.int32).tobytes()
    z, lengths = gifti._deflate(raw, 1)
    assert lengths is not None and len(lengths) > 8
    text = base64.b64encode(z)
    got, check = _decode(text, True, len(raw), lengths)
    assert got == raw and check == zlib.adler32(raw)
    # an index that does not sum to the stream is ignored (one inflate)
    assert _decode(text, True, len(raw), lengths[:-1] + [lengths[-1] + 1])[0] == raw
    # an index that sums to the stream but splits it elsewhere fails a chunk
    with pytest.raises(ValueError):
        _decode(text, True, len(raw), [lengths[0] - 3, lengths[1] + 3] + lengths[2:])
    # a chunk whose data is damaged fails its own inflate or the combined check
    damaged = bytearray(z)
    at = 2 + lengths[0] + lengths[1] // 2
    damaged[at:at + 4] = b"\x00\x00\x00\x00"
    with pytest.raises(ValueError):
        _decode(base64.b64encode(bytes(damaged)), True, len(raw), lengths)
    # the array size decides the last chunk's length; another size is refused
    with pytest.raises(ValueError):
        _decode(text, True, len(raw) - 4, lengths)


def test_concurrent_decodes_agree(native_library):
    """Files decoded side by side share the helper-thread budget and give the same bytes."""

    from concurrent.futures import ThreadPoolExecutor

    from cat_surface_gpu_b200 import gifti

    arrays = [np.random.default_rng(k).integers(0, 1000, size=400_000, dtype=np.int32).tobytes() for k in range(6)]
    streams = [gifti._deflate(raw, 1) for raw in arrays]
    with ThreadPoolExecutor(6) as pool:
        got = list(pool.map(lambda k: _decode(base64.b64encode(streams[k][0]), True, len(arrays[k]),
                                              streams[k][1])[0], range(6)))
    assert got == arrays
