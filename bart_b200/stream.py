"""Reading the reference's array streams (src/misc/stream.c,
src/misc/stream_protocol.c), so that slices or frames of k-space arriving
over a pipe are reconstructed as they arrive.

A stream starts with a text header ``# Header\\n<size>\\n`` followed by the
.cfl header lines (``# Dimensions``, and ``# Data <file>`` when the data
live in a shared file instead of the stream itself), padded to <size>
bytes (write_stream_header, src/misc/io.c:429-468). Then come fixed-size
messages of MSG_HDR_SIZE = 24 bytes: ``\\n# <keyword>\\n<number>`` padded
with spaces (stream_encode, src/misc/stream_protocol.c). The settings are
``flags`` (the streamed dims, a bitmask), optionally ``binary`` (the data
travel inline) and a break ``---`` (stream_write_settings,
src/misc/stream.c:1146-1170). Each slice is then ``index <i>`` (the position
over the streamed dims, the first one fastest: md_unravel_index), optional
``block <n>`` events (n bytes that follow; ignored here), with binary
streams ``raw <n>`` followed by the slice's n bytes (its non-streamed dims in
column-major order, get_transport_layout, src/misc/stream.c:661-689), and a
break. Shared-file streams only announce an index; the slice is then read
from the data file.
"""

from __future__ import annotations

import numpy as np

from .cfl import DIMS

MSG_HDR_SIZE = 24


class StreamError(RuntimeError):
    pass


def _read_exact(f, n: int) -> bytes:
    b = b""
    while len(b) < n:
        c = f.read(n - len(b))
        if not c:
            break
        b += c
    return b


def _decode(msg: bytes):
    """(keyword, number or None, ext) of one message (stream_decode)."""
    if len(msg) != MSG_HDR_SIZE or not msg.startswith(b"\n# "):
        raise StreamError(f"bad stream message {msg!r}")
    body = msg[3:].split(b"\x00", 1)[0]
    kw, _, rest = body.partition(b"\n")
    num = rest.strip()
    return kw.decode(), (int(num) if num else None), msg[-1:] == b"\n"


class StreamReader:
    """An input stream (a binary file object, e.g. sys.stdin.buffer).
    ``dims`` (16), ``flags``, ``binary``; iterating yields (index, pos,
    block): pos the index unravelled over the streamed dims, block the
    slice (streamed dims of size 1) as an F-ordered complex64 array."""

    def __init__(self, f):
        self.f = f
        head = _read_exact(f, 13)		# "# Header\n" + 3 digits + "\n"
        if not head.startswith(b"# Header\n"):
            raise StreamError("not a stream: no '# Header'")
        size = int(head[9:].split(b"\n", 1)[0])
        text = (head + _read_exact(f, size - len(head))).decode("ascii", "replace")
        lines = text.split("\n")
        self.dims, self.datafile = None, None
        for i, ln in enumerate(lines):
            if ln == "# Dimensions":
                d = [int(v) for v in lines[i + 1].split()]
                self.dims = (d + [1] * DIMS)[:DIMS]
            elif ln == "# Data":
                self.datafile = lines[i + 1].strip()
        if self.dims is None:
            raise StreamError("stream header without dimensions")
        self.flags, self.binary = None, False
        while True:	# stream_read_settings
            kw, num, _ = _decode(_read_exact(f, MSG_HDR_SIZE))
            if kw == "flags":
                self.flags = num
            elif kw == "binary":
                self.binary = True
            elif kw == "---":
                break
            else:
                raise StreamError(f"unexpected '{kw}' in the stream settings")
        if self.flags is None:
            raise StreamError("stream without flags")
        self.sdims = [d for d in range(DIMS) if self.flags & (1 << d)]
        self.slice_dims = [1 if (self.flags & (1 << d)) else n for d, n in enumerate(self.dims)]
        self.total = int(np.prod([self.dims[d] for d in self.sdims]))
        self._data = None
        if not self.binary:
            if not self.datafile:
                raise StreamError("shared-memory stream without a data file")
            self._data = np.memmap(self.datafile, dtype=np.complex64, mode="r", shape=tuple(self.dims), order="F")

    def position(self, index: int) -> tuple:
        """md_unravel_index over the streamed dims, the first one fastest."""
        pos = []
        for d in self.sdims:
            pos.append(index % self.dims[d])
            index //= self.dims[d]
        return tuple(pos)

    def __iter__(self):
        nbytes = 8 * int(np.prod(self.slice_dims))
        while True:
            m = _read_exact(self.f, MSG_HDR_SIZE)
            if not m:
                return		# the writer closed the stream
            kw, index, _ = _decode(m)
            if kw != "index" or index is None or not (0 <= index < self.total):
                raise StreamError(f"expected an index, got '{kw}' {index}")
            raw = None
            while True:
                kw, num, _ = _decode(_read_exact(self.f, MSG_HDR_SIZE))
                if kw == "---":
                    break
                if kw in ("raw", "block"):
                    payload = _read_exact(self.f, num)
                    if len(payload) != num:
                        raise StreamError("stream ended inside a data message")
                    if kw == "raw":
                        raw = payload
                else:
                    raise StreamError(f"unexpected '{kw}' in slice {index}")
            pos = self.position(index)
            if self.binary:
                if raw is None or len(raw) != nbytes:
                    raise StreamError(f"slice {index}: {0 if raw is None else len(raw)} bytes, {nbytes} expected")
                block = np.frombuffer(raw, dtype=np.complex64).reshape(self.slice_dims, order="F")
            else:
                sl = [slice(None)] * DIMS
                for d, p in zip(self.sdims, pos):
                    sl[d] = slice(p, p + 1)
                block = np.asarray(self._data[tuple(sl)])
            yield index, pos, np.asfortranarray(block)
