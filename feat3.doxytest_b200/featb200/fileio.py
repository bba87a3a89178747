"""The reference's container file formats for the containers of this path.

Binary formats (`FileMode::fm_csr` for SparseMatrixCSR, `fm_dv` for DenseVector, also written for
`fm_binary`) are the uncompressed form of the reference's container serialisation
(kernel/lafem/container.hpp:440-600, `_serialize`; reading `_deserialize`:622-775), always stored
with double values and 64-bit indices (sparse_matrix_csr.hpp:1066-1069, dense_vector.hpp:716-718):

    u64[0]   total bytes (= payload + 16 bytes of zero padding)
    u64[1]   file mode (fm_dv = 1, fm_csr = 4; kernel/lafem/base.hpp:31-47)
    u64[2,3] feature hashes of the value and index types: size | int << 32 | float << 33 | signed << 34
    u64[4..9] counts: element arrays, index arrays, element sizes, index sizes, scalar indices, scalar
             values; u64[10] compression mode (0x11 = elements off | indices off; base.hpp:96-110)
    then per element array its length and byte size, per index array its length and byte size, the
    scalar indices (container size, then rows, columns, used elements for CSR), the element arrays
    (CSR: val), the index arrays (CSR: col_ind, row_ptr), 16 zero bytes.

ASCII formats: Matrix Market coordinate (`fm_mtx`, 1-based, values in C++ `std::scientific`, i.e.
six digits: lossy), Matrix Market array for vectors, and one `std::scientific` value per line
(`fm_exp`).  Compressed binary files (zlib / zfp) are rejected: the reference needs third-party
libraries for them.
"""
from __future__ import annotations

import struct

import numpy as np

FM_DV = 1
FM_CSR = 4
COMPRESSION_OFF = 0x11   # elements_off | indices_off
_ELEMENTS_MASK, _INDICES_MASK = 0xF0, 0x0F
HASH_F64 = 8 | (1 << 33) | (1 << 34)
HASH_U64 = 8 | (1 << 32)


def _header(mode, elements, indices, scalars):
    words = [0, mode, HASH_F64, HASH_U64, len(elements), len(indices), len(elements), len(indices), len(scalars), 0,
             COMPRESSION_OFF]
    words += [a.size for a in elements] + [a.size * 8 for a in elements]
    words += [a.size for a in indices] + [a.size * 8 for a in indices]
    words += list(scalars)
    return words


def _serialize(mode, elements, indices, scalars):
    elements = [np.ascontiguousarray(a, dtype="<f8") for a in elements]
    indices = [np.ascontiguousarray(a, dtype="<u8") for a in indices]
    words = _header(mode, elements, indices, scalars)
    payload = 8 * len(words) + sum(a.nbytes for a in elements) + sum(a.nbytes for a in indices)
    words[0] = payload + 16
    return b"".join([struct.pack(f"<{len(words)}Q", *words)] + [a.tobytes() for a in elements] +
                    [a.tobytes() for a in indices] + [bytes(16)])


def _deserialize(mode, data):
    w = np.frombuffer(data, dtype="<u8", count=11)
    if int(w[1]) != mode:
        raise ValueError(f"file mode {int(w[1])} is not the expected {mode}")
    comp = int(w[10])
    if (comp & _ELEMENTS_MASK) not in (0x00, 0x10) or (comp & _INDICES_MASK) not in (0x0, 0x1):
        raise ValueError("compressed container files (zlib/zfp) are not supported")
    for h, want in ((int(w[2]), HASH_F64), (int(w[3]), None)):
        if want is not None and (h >> 32) != (want >> 32):
            raise ValueError("value type of the file is not floating point")
    vsize, isize = int(w[2]) & 0xFFFFFFFF, int(w[3]) & 0xFFFFFFFF
    ne, ni, ns, nd = int(w[6]), int(w[7]), int(w[8]), int(w[9])
    k = 11
    hdr = np.frombuffer(data, dtype="<u8", count=k + 2 * ne + 2 * ni + ns)
    esz = [int(x) for x in hdr[k:k + ne]]
    k += 2 * ne
    isz = [int(x) for x in hdr[k:k + ni]]
    k += 2 * ni
    scal = [int(x) for x in hdr[k:k + ns]]
    k += ns
    off = 8 * k + nd * vsize
    vdt = {8: "<f8", 4: "<f4"}[vsize]
    idt = {8: "<u8", 4: "<u4"}[isize]
    elements = []
    for n in esz:
        elements.append(np.frombuffer(data, dtype=vdt, count=n, offset=off).astype(np.float64))
        off += n * vsize
    indices = []
    for n in isz:
        indices.append(np.frombuffer(data, dtype=idt, count=n, offset=off).astype(np.uint64))
        off += n * isize
    return elements, indices, scal


# ------------------------------------------------------------------------------ CSR matrices
def write_csr(path, rows, columns, row_ptr, col_ind, val, mode="csr"):
    if mode in ("csr", "binary"):
        nnz = int(np.asarray(val).size)
        data = _serialize(FM_CSR, [val], [col_ind, row_ptr], [rows * columns, rows, columns, nnz])
        with open(path, "wb") as f:
            f.write(data)
    elif mode == "mtx":
        rp = np.asarray(row_ptr, dtype=np.int64)
        ci = np.asarray(col_ind, dtype=np.int64)
        v = np.asarray(val, dtype=np.float64)
        with open(path, "w") as f:
            f.write("%%MatrixMarket matrix coordinate real general\n")
            f.write(f"{rows} {columns} {v.size}\n")
            for r in range(rows):
                for j in range(rp[r], rp[r + 1]):
                    f.write(f"{r + 1} {ci[j] + 1} {v[j]:e}\n")
    else:
        raise ValueError(f"unsupported file mode {mode!r}")


def read_csr(path, mode="csr"):
    """(rows, columns, row_ptr, col_ind, val) with uint64 indices and float64 values."""
    if mode in ("csr", "binary"):
        with open(path, "rb") as f:
            data = f.read()
        (val,), (col_ind, row_ptr), scal = _deserialize(FM_CSR, data)
        return scal[1], scal[2], row_ptr, col_ind, val
    if mode == "mtx":
        with open(path) as f:
            head = f.readline()
            if "coordinate real general" not in head and "coordinate real symmetric" not in head:
                raise ValueError("not a Matrix Market coordinate real file")
            sym = "symmetric" in head
            line = f.readline()
            while line.lstrip().startswith("%"):
                line = f.readline()
            rows, cols, _ = (int(t) for t in line.split()[:3])
            entries = {}
            for line in f:
                t = line.split()
                if len(t) < 3:
                    continue
                r, c, v = int(t[0]) - 1, int(t[1]) - 1, float(t[2])
                entries[(r, c)] = v
                if sym and r != c:
                    entries[(c, r)] = v
        keys = sorted(entries)
        row_ptr = np.zeros(rows + 1, dtype=np.uint64)
        for r, _c in keys:
            row_ptr[r + 1] += 1
        row_ptr = np.cumsum(row_ptr, dtype=np.uint64)
        col_ind = np.array([c for _r, c in keys], dtype=np.uint64)
        val = np.array([entries[k] for k in keys], dtype=np.float64)
        return rows, cols, row_ptr, col_ind, val
    raise ValueError(f"unsupported file mode {mode!r}")


# ------------------------------------------------------------------------------ dense vectors
def write_dv(path, elements, mode="dv"):
    v = np.ascontiguousarray(elements, dtype=np.float64)
    if mode in ("dv", "binary"):
        with open(path, "wb") as f:
            f.write(_serialize(FM_DV, [v], [], [v.size]))
    elif mode == "mtx":
        with open(path, "w") as f:
            f.write("%%MatrixMarket matrix array real general\n")
            f.write(f"{v.size} 1\n")
            f.writelines(f"{x:e}\n" for x in v)
    elif mode == "exp":
        with open(path, "w") as f:
            f.writelines(f"{x:e}\n" for x in v)
    else:
        raise ValueError(f"unsupported file mode {mode!r}")


def read_dv(path, mode="dv"):
    if mode in ("dv", "binary"):
        with open(path, "rb") as f:
            data = f.read()
        (v,), _, _ = _deserialize(FM_DV, data)
        return v
    if mode == "mtx":
        with open(path) as f:
            head = f.readline()
            if "array real general" not in head:
                raise ValueError("not a Matrix Market array file")
            line = f.readline()
            while line.lstrip().startswith("%"):
                line = f.readline()
            n = int(line.split()[0])
            return np.array([float(f.readline()) for _ in range(n)])
    if mode == "exp":
        with open(path) as f:
            return np.array([float(t) for t in f if t.strip()])
    raise ValueError(f"unsupported file mode {mode!r}")
