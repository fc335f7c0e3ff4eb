"""Self-contained GIFTI surface codec (two-array point/triangle files).

The reference reads and writes GIFTI through nibabel
(``src/cat_surface_gpu/gpu_pipeline.py:52-110``: ``read_gifti_mesh`` and
``write_gifti_mesh``).  This module keeps the same two public functions and the
same ``GiftiMesh`` record, but is written on the standard library only
(``xml.etree``, ``base64``, ``zlib``) so the package has no nibabel dependency.

Supported encodings on read: ``ASCII``, ``Base64Binary`` and
``GZipBase64Binary`` with little- or big-endian payloads and row- or
column-major ordering.  Writes always use ``GZipBase64Binary`` little-endian,
which is what CAT-Surface's gifticlib produces and accepts.
"""

from __future__ import annotations

import base64
from collections import OrderedDict
import ctypes
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
import os
from pathlib import Path
import threading
import xml.etree.ElementTree as ET
import zlib

import numpy as np

_DTYPES = {
    "NIFTI_TYPE_FLOAT32": np.float32,
    "NIFTI_TYPE_FLOAT64": np.float64,
    "NIFTI_TYPE_INT32": np.int32,
    "NIFTI_TYPE_UINT8": np.uint8,
    "NIFTI_TYPE_INT16": np.int16,
    "NIFTI_TYPE_INT64": np.int64,
}
_INTENT_CODES = {
    "NIFTI_INTENT_POINTSET": 1008,
    "NIFTI_INTENT_TRIANGLE": 1009,
}
_INTENT_NAMES = {value: key for key, value in _INTENT_CODES.items()}


@dataclass(frozen=True)
class GiftiMesh:
    """One GIFTI surface: float32 vertices ``[n, 3]`` and int32 faces ``[m, 3]``."""

    vertices: np.ndarray
    faces: np.ndarray

    def check(self, label: str = "mesh") -> "GiftiMesh":
        """``ValueError`` unless the vertices are finite and every face index names a vertex.

        The GPU kernels trust both, so a surface with NaN or infinite
        coordinates, or faces outside ``[0, n)``, is refused on the host.
        """

        check_vertices(self.vertices, label)
        faces = np.asarray(self.faces)
        if faces.ndim != 2 or faces.shape[1] != 3:
            raise ValueError(f"{label}: faces must have shape [m, 3], got {faces.shape}")
        n = int(np.asarray(self.vertices).shape[0])
        if faces.size and (int(faces.min()) < 0 or int(faces.max()) >= n):
            raise ValueError(f"{label}: a face index lies outside [0, {n})")
        return self


def check_vertices(vertices, label: str = "vertices") -> None:
    """``ValueError`` unless ``vertices`` is a non-empty ``[n, 3]`` array of finite numbers."""

    values = np.asarray(vertices)
    if values.ndim != 2 or values.shape[1] != 3 or values.shape[0] == 0:
        raise ValueError(f"{label}: vertices must have shape [n, 3] with n > 0, got {values.shape}")
    if not np.isfinite(values).all():
        raise ValueError(f"{label}: vertices must be finite (NaN or infinite coordinates found)")


# Deflate of large arrays runs in parallel chunks (as pigz does): each chunk is a raw
# deflate stream ended by a sync flush (the last one by the final block), so their
# concatenation behind a zlib header and the Adler-32 of the whole input is one valid
# zlib stream that any inflater reads back as the same bytes.
_CHUNK = 1 << 17
_PARALLEL_MIN = 1 << 19
_POOL: ThreadPoolExecutor | None = None
_POOL_LOCK = threading.Lock()


def _pool() -> ThreadPoolExecutor:
    global _POOL
    with _POOL_LOCK:
        if _POOL is None:
            _POOL = ThreadPoolExecutor(max_workers=max(2, min(16, os.cpu_count() or 2)),
                                       thread_name_prefix="gifti-deflate")
    return _POOL


def _deflate(raw: bytes, level: int = 1) -> tuple[bytes, list[int] | None]:
    """zlib stream of ``raw`` and, when it was deflated in chunks, the chunks' compressed lengths."""

    if level == 0 or len(raw) < _PARALLEL_MIN:
        return zlib.compress(raw, level), None
    chunks = [raw[i: i + _CHUNK] for i in range(0, len(raw), _CHUNK)]
    last = len(chunks) - 1

    def one(item):
        index, chunk = item
        stream = zlib.compressobj(level, zlib.DEFLATED, -15)
        return stream.compress(chunk) + stream.flush(zlib.Z_FINISH if index == last else zlib.Z_SYNC_FLUSH)

    parts = list(_pool().map(one, enumerate(chunks)))
    header = bytes((0x78, 0x01 if level <= 1 else (0x5E if level <= 5 else (0x9C if level == 6 else 0xDA))))
    return header + b"".join(parts) + zlib.adler32(raw).to_bytes(4, "big"), [len(part) for part in parts]


# The chunk index of a payload deflated here rides in the array's MetaData, so a reader
# can inflate the chunks in parallel: each is an independent raw deflate stream.  Other
# readers ignore the entry and inflate the one zlib stream as usual.
_CHUNK_KEY = "DeflateChunkLengths"


def _chunk_metadata(lengths: list[int] | None) -> str:
    if not lengths:
        return "<MetaData/>\n"
    value = f"{_CHUNK}:" + ",".join(str(n) for n in lengths)
    return f"<MetaData><MD><Name><![CDATA[{_CHUNK_KEY}]]></Name><Value><![CDATA[{value}]]></Value></MD></MetaData>\n"


def _chunk_lengths(element: ET.Element) -> list[int] | None:
    meta = element.find("MetaData")
    if meta is None:
        return None
    for md in meta.findall("MD"):
        name, value = md.find("Name"), md.find("Value")
        if name is not None and (name.text or "").strip() == _CHUNK_KEY and value is not None and value.text:
            size, _, lengths = value.text.strip().partition(":")
            try:
                if int(size) != _CHUNK:
                    return None
                return [int(n) for n in lengths.split(",")]
            except ValueError:
                return None
    return None


def _decode_payload(payload: bytes, gzip: bool, lengths: list[int] | None, out: np.ndarray) -> int:
    """Decode base64 ``payload`` (inflating it when ``gzip``) into the bytes of ``out``; returns their Adler-32.

    Runs in the native library without the interpreter lock (the chunks of a
    chunk-indexed stream on several threads); ``ValueError`` when the payload
    is not base64, the stream is corrupt or truncated (Adler-32 checked as
    zlib does), or it decodes to another size than ``out``.  An index that
    does not fit the stream is ignored and the stream inflates as one.
    """

    from . import _native

    index = (ctypes.c_longlong * len(lengths))(*lengths) if lengths else None
    check = ctypes.c_uint(0)
    status = _native.library().csg_gifti_decode(payload, len(payload), int(bool(gzip)), index,
                                                len(lengths) if lengths else 0, _CHUNK, out.ctypes.data, out.nbytes,
                                                ctypes.byref(check))
    if status != _native.CSG_OK:
        raise ValueError(_native.last_error())
    return check.value


# Encoded payloads of the int32 arrays decoded most recently (face arrays): writing an
# array with the same bytes reuses its payload instead of compressing it again.  Keyed
# by (DataType, shape, Adler-32 of the bytes) -- the check value a zlib stream carries,
# so a read gets it for free; a hit is confirmed by comparing the bytes themselves.
_PAYLOADS: OrderedDict = OrderedDict()
_PAYLOADS_MAX = 8
_PAYLOADS_LOCK = threading.Lock()


def _remember_payload(dtype_name: str, shape: tuple, raw: bytes, check: int, payload: bytes,
                      lengths: list[int] | None) -> None:
    key = (dtype_name, shape, check)
    with _PAYLOADS_LOCK:
        _PAYLOADS[key] = (raw, payload, lengths)
        _PAYLOADS.move_to_end(key)
        while len(_PAYLOADS) > _PAYLOADS_MAX:
            _PAYLOADS.popitem(last=False)


def _known_payload(dtype_name: str, shape: tuple, raw: bytes) -> tuple[bytes, list[int] | None] | None:
    with _PAYLOADS_LOCK:
        hit = _PAYLOADS.get((dtype_name, shape, zlib.adler32(raw)))
    if hit is not None and hit[0] == raw:
        return hit[1], hit[2]
    return None


def _decode_array(element: ET.Element, payloads: list[bytes] = ()) -> tuple[np.ndarray, int]:
    attrs = element.attrib
    dtype_name = attrs.get("DataType", "NIFTI_TYPE_FLOAT32")
    if dtype_name not in _DTYPES:
        raise ValueError(f"Unsupported GIFTI DataType {dtype_name}")
    dtype = np.dtype(_DTYPES[dtype_name])
    dims = int(attrs.get("Dimensionality", "1"))
    shape = tuple(int(attrs[f"Dim{i}"]) for i in range(dims))
    encoding = attrs.get("Encoding", "ASCII")
    endian = attrs.get("Endian", "LittleEndian")
    order = "F" if attrs.get("ArrayIndexingOrder", "RowMajorOrder") == "ColumnMajorOrder" else "C"
    count = int(np.prod(shape)) if shape else 0
    if encoding == "ASCII":
        data_element = element.find("Data")
        text = "" if data_element is None or data_element.text is None else data_element.text
        values = np.array(text.split(), dtype=np.float64 if dtype.kind == "f" else np.int64)
        values = values.astype(dtype)
        if values.size != count:
            raise ValueError(f"GIFTI array holds {values.size} values, header says {count}")
    elif encoding in ("Base64Binary", "GZipBase64Binary"):
        payload = _payload(element, payloads)
        gzip = encoding == "GZipBase64Binary"
        lengths = _chunk_lengths(element) if gzip else None
        out = np.empty(count * dtype.itemsize, dtype=np.uint8)
        check = _decode_payload(payload, gzip, lengths, out)
        if gzip and dtype_name == "NIFTI_TYPE_INT32" and endian == "LittleEndian" and order == "C":
            _remember_payload(dtype_name, shape, out.tobytes(), check, _without_whitespace(payload), lengths)
        wire = dtype.newbyteorder("<" if endian == "LittleEndian" else ">")
        values = out.view(wire).astype(dtype, copy=False)
    else:
        raise ValueError(f"Unsupported GIFTI encoding {encoding}")
    intent_attr = attrs.get("Intent", "NIFTI_INTENT_NONE")
    intent = _INTENT_CODES.get(intent_attr, 0)
    return np.ascontiguousarray(values.reshape(shape, order=order)), intent


_BASE64_BYTES = frozenset(b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/=")


def _parse_document(data: bytes) -> tuple[ET.Element, list[bytes]]:
    """The GIFTI document's element tree and its encoded payloads, cut out before parsing.

    Every ``<Data>`` payload that is plain base64 text (no markup, entities or
    CDATA) is replaced by a placeholder ``@k@``, the rest of the document -- a
    few kilobytes -- is parsed by ElementTree (so the document is still
    checked for well-formedness), and payload ``k`` is returned as bytes for
    :func:`_payload`.  Parsing the megabytes of payload text was most of a
    mesh read.
    """

    pieces, payloads, at = [], [], 0
    while True:
        start = data.find(b"<Data>", at)
        if start < 0:
            break
        # the first '<' after the tag ends a payload without markup (a byte search, far
        # faster than one for the whole closing tag); anything else takes the full parse
        end = data.find(b"<", start + 6)
        if end < 0:
            break
        payload = data[start + 6:end]
        if not data.startswith(b"</Data>", end) or len(payload) < 4096 \
                or not _BASE64_BYTES.issuperset(payload[:8192].translate(None, b" \t\r\n")[:4096]) or b"&" in payload:
            pieces.append(data[at:end])
            at = end
            continue
        pieces.append(data[at:start + 6])
        pieces.append(b"@%d@" % len(payloads))
        payloads.append(payload)
        at = end
    pieces.append(data[at:])
    return ET.fromstring(b"".join(pieces)), payloads


def _payload(element: ET.Element, payloads: list[bytes]) -> bytes:
    """The encoded text of a DataArray's Data element, as bytes (a cut-out payload or the parsed text)."""

    data = element.find("Data")
    text = "" if data is None or data.text is None else data.text
    if payloads and text.startswith("@") and text.endswith("@") and text[1:-1].isdigit():
        index = int(text[1:-1])
        if index < len(payloads):
            return payloads[index]
    return text.encode("utf-8")


def _without_whitespace(payload: bytes) -> bytes:
    if any(c in payload for c in (b" ", b"\t", b"\r", b"\n")):
        return payload.translate(None, b" \t\r\n")
    return payload


def read_gifti_arrays(path: str | Path) -> list[tuple[np.ndarray, int]]:
    """Return every data array of a GIFTI file with its NIfTI intent code.

    A file that is not well-formed XML, or whose array payload does not
    decode (bad base64, a truncated or corrupt zlib stream, a size that
    disagrees with the header), raises ``ValueError``.
    """

    try:
        root, payloads = _parse_document(Path(path).read_bytes())
    except ET.ParseError as error:
        raise ValueError(f"Not a GIFTI file (XML: {error}): {path}") from error
    if root.tag != "GIFTI":
        raise ValueError(f"Not a GIFTI file: {path}")
    try:
        return [_decode_array(item, payloads) for item in root.findall("DataArray")]
    except (zlib.error, KeyError, TypeError) as error:
        raise ValueError(f"Corrupt GIFTI data array ({error}): {path}") from error
    except ValueError as error:
        raise ValueError(f"Corrupt GIFTI data array ({error}): {path}") from error


def read_gifti_mesh(path: str | Path) -> GiftiMesh:
    """Read the first point-set and triangle arrays of a GIFTI surface.

    Mirrors ``read_gifti_mesh`` of the reference (``gpu_pipeline.py:52-71``):
    ``ValueError`` when fewer than two arrays are present or when either array
    is not ``[*, 3]``.
    """

    arrays = read_gifti_arrays(path)
    if len(arrays) < 2:
        raise ValueError(f"GIFTI file must contain vertex and face arrays: {path}")
    vertices = arrays[0][0]
    faces = arrays[1][0]
    if vertices.ndim != 2 or vertices.shape[1] != 3:
        raise ValueError(f"Vertex array must have shape [n, 3]: {path} -> {vertices.shape}")
    if faces.ndim != 2 or faces.shape[1] != 3:
        raise ValueError(f"Face array must have shape [m, 3]: {path} -> {faces.shape}")
    return GiftiMesh(
        vertices=np.ascontiguousarray(vertices, dtype=np.float32),
        faces=np.ascontiguousarray(faces, dtype=np.int32),
    )


def _encode_array(values: np.ndarray, intent: int, dtype_name: str,
                  stored: tuple[bytes, list[int] | None] | None = None) -> list[bytes]:
    """One DataArray, as pieces of the document; ``stored`` is a (payload, chunk lengths) pair to write as it is."""

    if stored is None:
        raw = np.ascontiguousarray(values).astype(values.dtype.newbyteorder("<")).tobytes()
        stored = _known_payload(dtype_name, tuple(values.shape), raw) if dtype_name == "NIFTI_TYPE_INT32" else None
        if stored is None:
            # index arrays: deflate level 1 (as small as level 6, 40% of the raw bytes, at a
            # fifth of the time); float32 coordinates barely compress (92% at level 1 for 25 ms
            # per 61k-vertex array), so they go in stored blocks, a zlib stream every reader
            # inflates, at a millisecond each way
            compressed, lengths = _deflate(raw, 0 if values.dtype.kind == "f" else 1)
            stored = base64.b64encode(compressed), lengths
    payload, lengths = stored
    dims = "".join(f' Dim{i}="{size}"' for i, size in enumerate(values.shape))
    intent_name = _INTENT_NAMES.get(intent, "NIFTI_INTENT_NONE")
    transform = ""
    if intent == _INTENT_CODES["NIFTI_INTENT_POINTSET"]:
        transform = (
            "<CoordinateSystemTransformMatrix>"
            "<DataSpace><![CDATA[NIFTI_XFORM_UNKNOWN]]></DataSpace>"
            "<TransformedSpace><![CDATA[NIFTI_XFORM_UNKNOWN]]></TransformedSpace>"
            "<MatrixData>1 0 0 0 0 1 0 0 0 0 1 0 0 0 0 1</MatrixData>"
            "</CoordinateSystemTransformMatrix>\n"
        )
    head = (
        f'<DataArray Intent="{intent_name}" DataType="{dtype_name}" '
        f'ArrayIndexingOrder="RowMajorOrder" Dimensionality="{values.ndim}"{dims} '
        'Encoding="GZipBase64Binary" Endian="LittleEndian" ExternalFileName="" ExternalFileOffset="">\n'
        + _chunk_metadata(lengths) + f"{transform}<Data>"
    )
    return [head.encode("ascii"), payload, b"</Data>\n</DataArray>\n"]


def write_gifti_mesh(
    path: str | Path,
    mesh: GiftiMesh,
    *,
    reference_path: str | Path | None = None,
) -> None:
    """Write vertices (float32) and faces (int32) as a two-array GIFTI file.

    Mirrors ``write_gifti_mesh`` of the reference (``gpu_pipeline.py:74-110``):
    array intents are copied from ``reference_path`` when it is given.
    """

    intents = None
    if reference_path is not None:
        intents = [_INTENT_CODES.get(item.attrib.get("Intent", "NIFTI_INTENT_NONE"), 0)
                   for item in _data_arrays(reference_path)[0]]
    _write_mesh(path, mesh, intents)


def _data_arrays(path) -> tuple[list[ET.Element], list[bytes]]:
    """The DataArray elements of a GIFTI file and its cut-out payloads, not decoded."""

    root, payloads = _parse_document(Path(path).read_bytes())
    if root.tag != "GIFTI":
        raise ValueError(f"Not a GIFTI file: {path}")
    return root.findall("DataArray"), payloads


def _shape(element: ET.Element) -> tuple[int, ...]:
    attrs = element.attrib
    return tuple(int(attrs[f"Dim{i}"]) for i in range(int(attrs.get("Dimensionality", "1"))))


def _verbatim_faces(element: ET.Element, payloads: list[bytes]) -> tuple[bytes, list[int] | None] | None:
    """The payload (and chunk index) of an [m, 3] int32 little-endian row-major gzip face array, as stored."""

    attrs = element.attrib
    shape = _shape(element)
    if (attrs.get("DataType") == "NIFTI_TYPE_INT32" and attrs.get("Encoding") == "GZipBase64Binary"
            and attrs.get("Endian", "LittleEndian") == "LittleEndian"
            and attrs.get("ArrayIndexingOrder", "RowMajorOrder") == "RowMajorOrder"
            and len(shape) == 2 and shape[1] == 3):
        payload = _without_whitespace(_payload(element, payloads))
        if payload:
            return payload, _chunk_lengths(element)
    return None


def _write_mesh(path, mesh: GiftiMesh, intents, faces_payload: tuple[bytes, list[int] | None] | None = None) -> None:
    point_intent = _INTENT_CODES["NIFTI_INTENT_POINTSET"]
    triangle_intent = _INTENT_CODES["NIFTI_INTENT_TRIANGLE"]
    if intents is not None:
        if len(intents) >= 1 and intents[0]:
            point_intent = intents[0]
        if len(intents) >= 2 and intents[1]:
            triangle_intent = intents[1]
    vertices = np.ascontiguousarray(mesh.vertices, dtype=np.float32)
    faces = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    if vertices.ndim != 2 or vertices.shape[1] != 3 or faces.ndim != 2 or faces.shape[1] != 3:
        raise ValueError("GIFTI mesh arrays must have shape [n, 3] and [m, 3]")
    document = b"".join([
        b'<?xml version="1.0" encoding="UTF-8"?>\n'
        b'<!DOCTYPE GIFTI SYSTEM "http://www.nitrc.org/frs/download.php/115/gifti.dtd">\n'
        b'<GIFTI Version="1.0" NumberOfDataArrays="2">\n<MetaData/>\n<LabelTable/>\n',
        *_encode_array(vertices, point_intent, "NIFTI_TYPE_FLOAT32"),
        *_encode_array(faces, triangle_intent, "NIFTI_TYPE_INT32", faces_payload),
        b"</GIFTI>\n",
    ])
    output = Path(path)
    output.parent.mkdir(parents=True, exist_ok=True)
    output.write_bytes(document)


def write_vertices_like(reference_path: str | Path, output_path: str | Path, vertices: np.ndarray) -> None:
    """Copy a GIFTI surface and replace its vertices; faces are byte-identical.

    Same contract as the reference's ``_write_vertices_like``
    (``surf2sphere.py:899-916``): topology is carried over from
    ``reference_path`` unchanged, so triangle arrays are exact by construction.
    """

    elements, payloads = _data_arrays(reference_path)
    if len(elements) < 2:
        raise ValueError(f"GIFTI file must contain vertex and face arrays: {reference_path}")
    values = np.ascontiguousarray(vertices, dtype=np.float32)
    if values.shape != _shape(elements[0]):
        raise ValueError(f"vertices shape {values.shape} does not match {_shape(elements[0])}")
    intents = [_INTENT_CODES.get(item.attrib.get("Intent", "NIFTI_INTENT_NONE"), 0) for item in elements]
    payload = _verbatim_faces(elements[1], payloads)
    if payload is not None:
        # the reference's own face payload, copied as stored: the same bytes without re-encoding
        faces = np.empty(_shape(elements[1]), dtype=np.int32)
    else:
        faces = np.ascontiguousarray(_decode_array(elements[1], payloads)[0], dtype=np.int32)
    _write_mesh(output_path, GiftiMesh(values, faces), intents, payload)
