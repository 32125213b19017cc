"""readMesh2dHDF5 (utilsIO.jl:107-252) without libhdf5.

The reference reads its meshes with HDF5.jl: 23 datasets (nCells, nNodes,
nNeibCells, nBSets, xNodes, yNodes, mesh_connectivity, bc_data, bc_indexes,
cell_nodes_X/Y, cell_mid_points, cell_areas, HX, cell_edges_Nx/Ny/length,
cell_stiffness, cell_clusters, node_stencils, node2cellL2up/down,
cells2nodes) in the root group, each a Julia column-major array written with
reversed HDF5 dimensions.  This module parses exactly the subset of the HDF5
file format those files use -- superblock versions 0-3, version 1 and 2
object headers, old-style (symbol table) and new-style (compact link
messages or fractal heap + version 2 B-tree) groups, contiguous and compact
dataset storage of fixed-point and IEEE floating-point data -- and raises on
anything else (chunked or filtered storage, other types).
"""
from __future__ import annotations

import struct
from typing import Dict, List, Tuple

import numpy as np

from .mesh import Mesh2d


class HDF5FormatError(ValueError):
    pass


class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        if data[:8] != b"\x89HDF\r\n\x1a\n":
            raise HDF5FormatError("not an HDF5 file")
        self.so = 8  # size of offsets
        self.sl = 8  # size of lengths
        ver = data[8]
        if ver in (0, 1):
            self.so, self.sl = data[13], data[14]
            base = 24 + (4 if ver == 1 else 0)
            # base address, free-space address, EOF address, driver info address
            p = base + 4 * self.so
            # root group symbol table entry
            self.root_oh = self.off(p + self.so)
        elif ver in (2, 3):
            self.so, self.sl = data[9], data[10]
            p = 12
            p += 3 * self.so  # base, superblock extension, EOF
            self.root_oh = self.off(p)
        else:
            raise HDF5FormatError(f"superblock version {ver}")

    # -- primitive reads ----------------------------------------------------
    def u(self, p: int, n: int) -> int:
        return int.from_bytes(self.d[p:p + n], "little")

    def off(self, p: int) -> int:
        return self.u(p, self.so)

    def ln(self, p: int) -> int:
        return self.u(p, self.sl)

    # -- object headers -------------------------------------------------------
    def messages(self, oh: int) -> List[Tuple[int, int, int]]:
        """(type, data offset, size) of every message of an object header."""
        d = self.d
        out = []
        if d[oh:oh + 4] == b"OHDR":
            ver, flags = d[oh + 4], d[oh + 5]
            p = oh + 6
            if flags & 0x20:
                p += 16
            if flags & 0x10:
                p += 4
            csize = 1 << (flags & 3)
            size0 = self.u(p, csize)
            p += csize
            blocks = [(p, size0)]
            track_order = bool(flags & 0x04)
            while blocks:
                s, ln = blocks.pop(0)
                q, end = s, s + ln
                while q + 4 <= end:
                    t, sz, _fl = d[q], self.u(q + 1, 2), d[q + 3]
                    q += 4 + (2 if track_order else 0)
                    if t == 0x10:
                        a, l2 = self.off(q), self.ln(q + self.so)
                        blocks.append((a + 4, l2 - 8))  # OCHK signature and checksum
                    out.append((t, q, sz))
                    q += sz
            return out
        if d[oh] != 1:
            raise HDF5FormatError(f"object header version {d[oh]} at {oh}")
        nmsg = self.u(oh + 2, 2)
        size0 = self.u(oh + 8, 4)
        blocks = [(oh + 16, size0)]
        while blocks and len(out) < nmsg:
            s, ln = blocks.pop(0)
            q = s
            while q < s + ln and len(out) < nmsg:
                t, sz = self.u(q, 2), self.u(q + 2, 2)
                body = q + 8
                if t == 0x10:
                    blocks.append((self.off(body), self.ln(body + self.so)))
                out.append((t, body, sz))
                q = body + sz
        return out

    # -- groups ---------------------------------------------------------------
    def links(self, oh: int) -> Dict[str, int]:
        msgs = self.messages(oh)
        res: Dict[str, int] = {}
        for t, p, sz in msgs:
            if t == 0x11:  # symbol table: v1 B-tree + local heap
                res.update(self._symbol_table(self.off(p), self.off(p + self.so)))
            elif t == 0x06:  # compact link message
                name, addr = self._link_message(p)
                if addr is not None:
                    res[name] = addr
            elif t == 0x02:  # link info: dense storage
                flags = self.d[p + 1]
                q = p + 2 + (8 if flags & 1 else 0)
                heap, name_bt = self.off(q), self.off(q + self.so)
                if heap != (1 << (8 * self.so)) - 1:
                    res.update(self._dense_links(heap, name_bt))
        return res

    def _symbol_table(self, btree: int, heap: int) -> Dict[str, int]:
        d = self.d
        if d[heap:heap + 4] != b"HEAP":
            raise HDF5FormatError("local heap signature")
        hdata = self.off(heap + 8 + 2 * self.sl)
        res = {}

        def walk(node):
            if d[node:node + 4] != b"TREE":
                raise HDF5FormatError("v1 B-tree signature")
            level, n = d[node + 5], self.u(node + 6, 2)
            p = node + 8 + 2 * self.so
            for _ in range(n):
                p += self.sl
                child = self.off(p)
                p += self.so
                if level > 0:
                    walk(child)
                else:
                    if d[child:child + 4] != b"SNOD":
                        raise HDF5FormatError("symbol node signature")
                    ns = self.u(child + 6, 2)
                    e = child + 8
                    for _ in range(ns):
                        noff, ohaddr = self.off(e), self.off(e + self.so)
                        s = hdata + noff
                        res[d[s:d.index(b"\0", s)].decode()] = ohaddr
                        e += 2 * self.so + 24
        walk(btree)
        return res

    def _link_message(self, p: int):
        d = self.d
        if d[p] != 1:
            raise HDF5FormatError("link message version")
        flags = d[p + 1]
        q = p + 2
        ltype = 0
        if flags & 0x08:
            ltype = d[q]
            q += 1
        if flags & 0x04:
            q += 8
        if flags & 0x10:
            q += 1
        nsz = 1 << (flags & 3)
        nlen = self.u(q, nsz)
        q += nsz
        name = d[q:q + nlen].decode()
        q += nlen
        if ltype != 0:
            return name, None  # soft / external links are not followed
        return name, self.off(q)

    def _dense_links(self, heap: int, btree: int) -> Dict[str, int]:
        d = self.d
        if d[heap:heap + 4] != b"FRHP":
            raise HDF5FormatError("fractal heap signature")
        p = heap + 5
        heap_id_len = self.u(p, 2)
        io_filter_len = self.u(p + 2, 2)
        hflags = d[p + 4]
        max_obj = self.u(p + 5, 4)
        # next huge id, huge-object B-tree, free space, free-space manager,
        # managed/allocated space, iterator, and the object counts and sizes
        p += 9 + 2 * self.so + 10 * self.sl
        width = self.u(p, 2)
        start_bs = self.ln(p + 2)
        max_dbs = self.ln(p + 2 + self.sl)
        max_heap_bits = self.u(p + 2 + 2 * self.sl, 2)
        root = self.off(p + 2 + 2 * self.sl + 4)
        cur_rows = self.u(p + 2 + 2 * self.sl + 4 + self.so, 2)
        if io_filter_len:
            raise HDF5FormatError("filtered fractal heap")
        offsize = (max_heap_bits + 7) // 8
        lensize = (min(max_dbs, max_obj).bit_length() + 7) // 8
        dblock_hdr = 5 + self.so + offsize + (4 if hflags & 2 else 0)
        # collect direct blocks: (heap offset of block start, file address, size)
        blocks = []

        def dblock(addr, size):
            if d[addr:addr + 4] != b"FHDB":
                raise HDF5FormatError("direct block signature")
            boff = self.u(addr + 5 + self.so, offsize)
            blocks.append((boff, addr, size))

        def iblock(addr, nrows):
            if d[addr:addr + 4] != b"FHIB":
                raise HDF5FormatError("indirect block signature")
            q = addr + 5 + self.so + offsize
            max_drows = (max_dbs.bit_length() - 1) - (start_bs.bit_length() - 1) + 2
            for r in range(nrows):
                bs = start_bs if r < 2 else start_bs << (r - 1)
                for _ in range(width):
                    child = self.off(q)
                    q += self.so
                    if child != (1 << (8 * self.so)) - 1 and child != 0:
                        if r < max_drows:
                            dblock(child, bs)
                        else:
                            irows = (bs.bit_length() - 1) - (start_bs.bit_length() - 1) - 1
                            iblock(child, max(irows, 0))

        if cur_rows == 0:
            dblock(root, start_bs)
        else:
            iblock(root, cur_rows)
        blocks.sort()

        def obj(heap_id: bytes) -> int:
            typ = (heap_id[0] >> 4) & 3
            if typ != 0:
                raise HDF5FormatError("only managed heap objects are supported")
            o = int.from_bytes(heap_id[1:1 + offsize], "little")
            for boff, addr, size in blocks:
                if boff <= o < boff + size:
                    return addr + (o - boff)
            raise HDF5FormatError("heap object outside the direct blocks")

        # v2 B-tree of link names (type 5 records: hash + heap id)
        if d[btree:btree + 4] != b"BTHD":
            raise HDF5FormatError("v2 B-tree signature")
        q = btree + 6
        rec_size = self.u(q + 4, 2)
        depth = self.u(q + 6, 2)
        root_addr = self.off(q + 10)
        root_n = self.u(q + 10 + self.so, 2)
        if depth != 0:
            # fall back to scanning every direct block's link messages
            return self._scan_blocks(blocks, dblock_hdr)
        if d[root_addr:root_addr + 4] != b"BTLF":
            raise HDF5FormatError("v2 B-tree leaf signature")
        res = {}
        r = root_addr + 6
        for _ in range(root_n):
            hid = d[r + 4:r + 4 + heap_id_len]
            name, addr = self._link_message(obj(hid))
            if addr is not None:
                res[name] = addr
            r += rec_size
        return res

    def _scan_blocks(self, blocks, hdr):
        res = {}
        for _boff, addr, size in blocks:
            q, end = addr + hdr, addr + size
            while q < end and self.d[q] == 1:
                name, a = self._link_message(q)
                flags = self.d[q + 1]
                nsz = 1 << (flags & 3)
                skip = 2 + (1 if flags & 8 else 0) + (8 if flags & 4 else 0) + (1 if flags & 16 else 0)
                nlen = self.u(q + skip, nsz)
                q += skip + nsz + nlen + self.so
                if a is not None:
                    res[name] = a
        return res

    # -- datasets -------------------------------------------------------------
    def dataset(self, oh: int) -> np.ndarray:
        dims = None
        dtype = None
        layout = None
        for t, p, sz in self.messages(oh):
            d = self.d
            if t == 0x01:
                ver, nd = d[p], d[p + 1]
                q = p + (8 if ver == 1 else 4)
                dims = [self.ln(q + self.sl * i) for i in range(nd)]
            elif t == 0x03:
                cls, size = d[p] & 0x0F, self.u(p + 4, 4)
                bf0 = d[p + 1]
                if bf0 & 1:
                    raise HDF5FormatError("big-endian data")
                if cls == 0:
                    dtype = np.dtype(("<i" if bf0 & 8 else "<u") + str(size))
                elif cls == 1:
                    dtype = np.dtype("<f" + str(size))
                else:
                    raise HDF5FormatError(f"datatype class {cls}")
            elif t == 0x08:
                ver, cl = d[p], d[p + 1]
                if ver != 3:
                    raise HDF5FormatError(f"layout message version {ver}")
                if cl == 0:
                    n = self.u(p + 2, 2)
                    layout = ("compact", p + 4, n)
                elif cl == 1:
                    layout = ("contiguous", self.off(p + 2), self.ln(p + 2 + self.so))
                else:
                    raise HDF5FormatError("chunked dataset storage")
            elif t == 0x0B:
                raise HDF5FormatError("filtered dataset")
        if dtype is None or layout is None:
            raise HDF5FormatError("dataset without type or layout")
        count = int(np.prod(dims)) if dims else 1
        raw = np.frombuffer(self.d, dtype=dtype, count=count, offset=layout[1])
        if not dims:
            return raw[0]
        # HDF5 dims are the reversed Julia dims of a column-major array
        return raw.reshape(tuple(reversed(dims)), order="F")


MESH_DATASETS = ("nCells", "nNodes", "nNeibCells", "nBSets", "xNodes", "yNodes", "mesh_connectivity", "bc_data",
                 "bc_indexes", "cell_nodes_X", "cell_nodes_Y", "cell_mid_points", "cell_areas", "HX", "cell_edges_Nx",
                 "cell_edges_Ny", "cell_edges_length", "cell_stiffness", "cell_clusters", "node_stencils",
                 "node2cellL2up", "node2cellL2down", "cells2nodes")


def read_datasets(path: str) -> Dict[str, np.ndarray]:
    with open(path, "rb") as f:
        data = f.read()
    r = _Reader(data)
    links = r.links(r.root_oh)
    return {name: r.dataset(addr) for name, addr in links.items()}


def readMesh2dHDF5(path: str) -> Mesh2d:
    """The reference's mesh reader (utilsIO.jl:107-252) -> Mesh2d."""
    if not path.endswith(".h5"):
        path = path + ".h5"
    ds = read_datasets(path)
    missing = [k for k in MESH_DATASETS if k not in ds]
    if missing:
        raise HDF5FormatError("mesh file lacks datasets: " + ", ".join(missing))
    return Mesh2d.from_arrays({k: ds[k] for k in MESH_DATASETS})
