"""The persisted autotuner store (csrc/tune_cache.cpp, on csrc/json.cpp) on the host: no GPU.

A small C++ driver compiled with g++ against tune_cache.cpp and json.cpp stores and reads picks:
round trip, a second key merged beside the first, a key replaced, members the store does
not own kept on rewrite, keys with quotes and backslashes, a missing file as a miss, and a
malformed file or entry refused with the PARSE prefix and left byte for byte as it was.
"""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "usermeso-2.0-mdpd_b200", "csrc")

DRIVER = r"""
#include "tune_cache.h"
#include <cstdio>
#include <cstring>
#include <stdexcept>
using namespace mdpd;
// driver put <path> <key> <density> <force> <ms> | get <path> <key>
int main(int argc, char **argv)
{
    try {
        if (argc == 7 && !std::strcmp(argv[1], "put")) {
            TunePick p;
            p.density = std::atoi(argv[4]);
            p.force = std::atoi(argv[5]);
            p.ms_per_step = std::atof(argv[6]);
            tune_cache_put(argv[2], argv[3], p);
            std::printf("stored\n");
        } else if (argc == 4 && !std::strcmp(argv[1], "get")) {
            TunePick p;
            if (tune_cache_get(argv[2], argv[3], p)) std::printf("hit %d %d %.3f\n", p.density, p.force, p.ms_per_step);
            else std::printf("miss\n");
        } else
            return 2;
    } catch (const std::exception &e) {
        std::printf("error %s\n", e.what());
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("tune")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "driver"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I" + CSRC, str(src), os.path.join(CSRC, "tune_cache.cpp"),
                    os.path.join(CSRC, "json.cpp"), "-o", str(exe)], check=True, capture_output=True, text=True)

    def run(*args):
        r = subprocess.run([str(exe)] + [str(a) for a in args], capture_output=True, text=True, check=True)
        return r.stdout.strip()
    return run


def test_round_trip_merge_and_replace(driver, tmp_path):
    f = tmp_path / "tune.json"
    k1 = "NVIDIA B200 sm148 | mdpd pair-once | rho 6.00 | rc 1.30 | particles 2^23 | boxes 2^8"
    k2 = "NVIDIA B200 sm148 | dpd full-list | rho 3.00 | rc 1.30 | particles 2^16 | boxes 2^0"
    assert driver("get", f, k1) == "miss"  # no file yet
    assert driver("put", f, k1, 6, 32, 7.78) == "stored"
    assert driver("get", f, k1) == "hit 6 32 7.780"
    assert driver("get", f, k2) == "miss"
    assert driver("put", f, k2, 2, 4, 0.5) == "stored"
    assert driver("get", f, k1) == "hit 6 32 7.780" and driver("get", f, k2) == "hit 2 4 0.500"
    assert driver("put", f, k1, 8, 32, 7.5) == "stored"
    assert driver("get", f, k1) == "hit 8 32 7.500"
    doc = json.loads(f.read_text())  # the file is plain JSON
    assert doc["version"] == 1 and list(doc["entries"]) == [k1, k2]
    assert doc["entries"][k2] == {"density": 2, "force": 4, "ms_per_step": 0.5}
    assert not [p for p in os.listdir(tmp_path) if ".tmp" in p]  # temporary renamed away


def test_foreign_members_kept_and_escaped_keys(driver, tmp_path):
    f = tmp_path / "tune.json"
    f.write_text(json.dumps({"note": "hand edited", "entries": {"old": {"density": 4, "force": 32, "x": [1, True, None]}},
                             "extra": {"a": "é"}}))
    key = 'weird "key" with \\ backslash'
    assert driver("put", f, key, 4, 32, 1.25) == "stored"
    doc = json.loads(f.read_text())
    assert doc["note"] == "hand edited" and doc["extra"] == {"a": "é"} and doc["version"] == 1
    assert doc["entries"]["old"] == {"density": 4, "force": 32, "x": [1, True, None]}
    assert driver("get", f, key) == "hit 4 32 1.250"
    assert driver("get", f, "old") == "hit 4 32 0.000"


@pytest.mark.parametrize("text", ["{", '{"entries": [1, 2]}', '[1, 2]', '{"entries": {"k": {"density": "six"}}}',
                                  '{"entries": {}} trailing', '{"a": 01x}'])
def test_malformed_file_refused_and_untouched(driver, tmp_path, text):
    f = tmp_path / "tune.json"
    f.write_text(text)
    out_get = driver("get", f, "k")
    out_put = driver("put", f, "k", 6, 32, 1.0)
    if text.startswith('{"entries": {"k"'):
        assert out_get.startswith("error PARSE: tune cache") and "density" in out_get
        assert out_put == "stored"  # a bad entry is replaced by a put of its key
        assert json.loads(f.read_text())["entries"]["k"]["density"] == 6
    else:
        assert out_get.startswith("error PARSE: tune cache"), out_get
        assert out_put.startswith("error PARSE: tune cache"), out_put
        assert f.read_text() == text
