"""The command line's file writers on the host (no GPU): the VTI written
from one dense block (header, UInt64 length words, scalar blocks, the
interleaved vector, footer), and the checkpoint with its sidecar, compiled
from the host sources into a small driver."""
import re
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HOST = ROOT / 'lbflow_b200' / 'csrc' / 'host'

DRIVER = r'''
#include "io.h"
#include <cstdio>
#include <string>
#include <vector>
int main(int argc, char** argv) {
    using namespace lbfhost;
    const std::string dir = argv[1];
    // 2 x 3 x 5 (z, y, x): density, then velocity (3 components).
    std::vector<std::size_t> sz = {2, 3, 5};
    const std::size_t N = 30;
    std::vector<double> d(4 * N);
    for (std::size_t i = 0; i < d.size(); ++i) d[i] = 0.25 * i - 3.0;
    writeVtiBlocks(dir + "/a.vti", sz, {"density"}, "velocity", 3, d.data());
    // Two-phase 2-D (y, x) = (4, 3): r0, r1, then v (2 components).
    std::vector<std::size_t> s2 = {4, 3};
    std::vector<double> c(4 * 12);
    for (std::size_t i = 0; i < c.size(); ++i) c[i] = 1.0 / (i + 1);
    writeVtiBlocks(dir + "/b.vti", s2, {"r0", "r1"}, "v", 2, c.data());
    std::vector<double> f(19 * N);
    for (std::size_t i = 0; i < f.size(); ++i) f[i] = i * 1e-3;
    writeCheckpoint(dir + "/field.0000000007.rst", f.data(), f.size());
    writeCheckpointMeta(dir + "/field.0000000007.rst", 7, 1, 3, 19, sz);
    validateCheckpoint(dir + "/field.0000000007.rst", 7, 1, 3, 19, sz);
    std::vector<double> back = readCheckpoint(dir + "/field.0000000007.rst", f.size());
    std::printf("%d\n", back == f ? 1 : 0);
    return 0;
}
'''


@pytest.fixture(scope='module')
def outputs(tmp_path_factory):
    d = tmp_path_factory.mktemp('io')
    (d / 'driver.cpp').write_text(DRIVER)
    exe = d / 'driver'
    subprocess.run(['g++', '-std=c++11', '-O1', '-I', str(HOST), '-o', str(exe), str(d / 'driver.cpp'),
                    str(HOST / 'io.cpp')], check=True)
    r = subprocess.run([str(exe), str(d)], capture_output=True, text=True, check=True)
    assert r.stdout.strip() == '1'
    return d


def blocks(path):
    data = path.read_bytes()
    head = data[:data.index(b'>_') + 2].decode()
    pos = len(head)
    out = []
    while not data[pos:].startswith(b'</AppendedData>'):
        n = struct.unpack_from('<Q', data, pos)[0]
        out.append(np.frombuffer(data, '<f8', n // 8, pos + 8))
        pos += 8 + n
    assert data[pos:] == b'</AppendedData></VTKFile>'
    return head, out


def test_vti_blocks_3d(outputs):
    head, (rho, vel) = blocks(outputs / 'a.vti')
    d = 0.25 * np.arange(120) - 3.0
    assert np.array_equal(rho, d[:30]) and np.array_equal(vel, d[30:])
    assert 'WholeExtent=" 0 4 0 2 0 1 "' in head            # x first, reference order reversed
    assert re.search(r'Name="velocity" NumberOfComponents="3" format="appended" offset="248"', head)


def test_vti_blocks_2d_two_phase(outputs):
    head, (r0, r1, v) = blocks(outputs / 'b.vti')
    c = 1.0 / (np.arange(48) + 1)
    assert np.array_equal(r0, c[:12]) and np.array_equal(r1, c[12:24]) and np.array_equal(v, c[24:])
    assert 'WholeExtent=" 0 2 0 3 0 0 "' in head and 'Scalars="r0 r1 "' in head


def test_checkpoint_and_sidecar(outputs):
    f = np.fromfile(outputs / 'field.0000000007.rst')
    assert np.array_equal(f, np.arange(570) * 1e-3)
    meta = (outputs / 'field.0000000007.rst.meta').read_text().splitlines()
    assert meta[0] == 'DRLAB_OUTGOING_V1' and meta[1] == '7 1 3 19' and meta[3] == 'NEXT_STREAM 8'
