"""Generate the golden fixtures under tests/golden/ (test infrastructure).

  python tests/golden/make_golden.py host
      TEA words from the reference's own premix_TEA (oracle/_ref/ref_pin host)
      -> tea_words.json; and the static-contact-angle deck's input data and density
      profiles from the reference tree -> static_contact_*.
  python tests/golden/make_golden.py device <ref_device.json>
      gaussian_TEA<4> values and nvcc contraction probes produced on a B200 by
      `oracle/_ref/ref_pin device <ref_device.json>` -> ref_device.json.
  python tests/golden/make_golden.py decks
      the reference's example input decks, verbatim -> decks/ (the quasi-2D pore deck is
      left out: its data file init_solids_fluids.dat is not in the reference tree)

Reads the reference tree at REF (default /root/reference); nothing at test time does.
"""
import gzip
import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("REF", "/root/reference")
DECK = os.path.join(REF, "examples/v2.5/static_contact_angle_in_a_slit_nano_channel")


def host():
    subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "REF=" + REF])
    subprocess.check_call([os.path.join(ROOT, "oracle/_ref/ref_pin"), "host",
                           os.path.join(HERE, "tea_words.json")])
    # deck input (9,280 atoms) and reference outputs, verbatim
    with open(os.path.join(DECK, "LAMMPS_init_noimage.dat"), "rb") as f, \
            gzip.open(os.path.join(HERE, "static_contact_init.dat.gz"), "wb", compresslevel=9) as g:
        shutil.copyfileobj(f, g)
    prof = {"deck": "examples/v2.5/static_contact_angle_in_a_slit_nano_channel/in.gpu.static_contact",
            "gpu": {}, "cpu": {}}
    for a in ("20", "30", "35"):
        rows = []
        with open(os.path.join(DECK, "out.profile.a_-" + a)) as f:
            for line in f:
                if line.strip():
                    y, c = line.split()
                    rows.append([float(y), float(c)])
        prof["gpu"]["-" + a] = rows
        rows = []
        with open(os.path.join(DECK, "CPU_simulations_to_match", "out.cpu.a-" + a)) as f:
            for line in f:
                t = line.split()
                if len(t) == 4 and not line.startswith("#"):
                    rows.append([float(t[1]), float(t[2])])
        prof["cpu"]["-" + a] = rows
    with open(os.path.join(HERE, "static_contact_profiles.json"), "w") as f:
        json.dump(prof, f, indent=1)


DECKS = {"box_10x10x10/in.test": "in.test",
         "liquid_vacuum_interface/in.gpu.water": "in.gpu.water",
         "static_contact_angle_in_a_slit_nano_channel/in.gpu.static_contact": "in.gpu.static_contact"}


def decks():
    os.makedirs(os.path.join(HERE, "decks"), exist_ok=True)
    for src, dst in DECKS.items():
        shutil.copyfile(os.path.join(REF, "examples/v2.5", src), os.path.join(HERE, "decks", dst))


def device(path):
    with open(path) as f:
        d = json.load(f)
    with open(os.path.join(HERE, "ref_device.json"), "w") as f:
        json.dump(d, f)


if __name__ == "__main__":
    if sys.argv[1] == "host":
        host()
    elif sys.argv[1] == "decks":
        decks()
    else:
        device(sys.argv[2])
