"""The self-contained HDF5 writer (pbpic_b200/csrc/h5_writer.h) on the CPU: a
small C++ program writes nested groups and datasets of every element type it
supports, and the test reader (tests/h5_reader.py, written from the published
file-format description) reads back every value."""
import os
import subprocess

import numpy as np

from h5_reader import read

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r'''
#include "h5_writer.h"
#include <vector>
#include <cstdio>
int main(int argc, char** argv) {
  std::vector<float> a(3 * 5);
  for (int i = 0; i < 15; ++i) a[i] = 0.5f * i - 3.0f;
  std::vector<double> d(7);
  for (int i = 0; i < 7; ++i) d[i] = 1.0 / (i + 1);
  std::vector<int32_t> k(4);
  for (int i = 0; i < 4; ++i) k[i] = -2 + 3 * i;
  std::vector<int64_t> q = {1ll << 40, -5};
  auto w = [](const void* p) { return [p](FILE* f, uint64_t n) { return fwrite(p, 1, n, f) == n; }; };
  h5w::Group root;
  root.datasets.push_back(h5w::Dataset{"floats", h5w::FLOAT, 4, {3, 5}, w(a.data())});
  root.datasets.push_back(h5w::Dataset{"doubles", h5w::FLOAT, 8, {7}, w(d.data())});
  root.datasets.push_back(h5w::Dataset{"ints", h5w::INT, 4, {4}, w(k.data())});
  for (int t = 0; t < 70; t += 10) {
    char name[16];
    snprintf(name, sizeof name, "%05d", t);
    h5w::Group g;
    g.name = name;
    g.datasets.push_back(h5w::Dataset{"longs", h5w::INT, 8, {2}, w(q.data())});
    g.datasets.push_back(h5w::Dataset{"spectra", h5w::INT, 4, {2, 2}, w(k.data())});
    root.groups.push_back(g);
  }
  h5w::Group empty;
  empty.name = "empty";
  root.groups.push_back(empty);
  std::string err;
  if (!h5w::write_file(argv[1], root, &err)) { fprintf(stderr, "%s\n", err.c_str()); return 1; }
  return 0;
}
'''


def test_writer_round_trip(tmp_path):
    src = tmp_path / "w.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "w"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "pbpic_b200", "csrc"), "-o", str(exe),
                    str(src)], check=True)
    out = tmp_path / "t.h5"
    subprocess.run([str(exe), str(out)], check=True)
    f = read(str(out))
    assert np.array_equal(f["floats"], (0.5 * np.arange(15) - 3.0).astype(np.float32).reshape(3, 5))
    assert f["floats"].dtype == np.float32
    assert np.array_equal(f["doubles"], 1.0 / np.arange(1, 8))
    assert np.array_equal(f["ints"], np.array([-2, 1, 4, 7], dtype=np.int32))
    for t in range(0, 70, 10):
        g = f[f"{t:05d}"]
        assert np.array_equal(g["longs"], np.array([1 << 40, -5], dtype=np.int64))
        assert np.array_equal(g["spectra"], np.array([[-2, 1], [4, 7]], dtype=np.int32))
    assert f["empty"] == {}
    assert sorted(f) == sorted(["floats", "doubles", "ints", "empty"] + [f"{t:05d}" for t in range(0, 70, 10)])
