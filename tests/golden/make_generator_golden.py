"""Record the reference generator's output for the shape fixtures.

Runs the reference scene generator, built from its own sources into
oracle/_ref/GeneratorForMph (make -C oracle ref), on every .boid file under
tests/golden/shapes/ and stores the SHA-256 of each .grid it writes in
tests/golden/golden.json under generator_kat["shapes/<name>"]:

    python tests/golden/make_generator_golden.py
"""
import glob
import hashlib
import json
import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
GEN = os.path.join(ROOT, "oracle", "_ref", "GeneratorForMph")


def main():
    path = os.path.join(HERE, "golden.json")
    with open(path) as f:
        gold = json.load(f)
    for boid in sorted(glob.glob(os.path.join(HERE, "shapes", "*.boid"))):
        name = os.path.splitext(os.path.basename(boid))[0]
        with tempfile.TemporaryDirectory() as tmp:
            shutil.copyfile(boid, os.path.join(tmp, name + ".boid"))
            # the generator reads <arg>.boid and writes <arg>.grid in the cwd
            subprocess.run([GEN, name], cwd=tmp, check=True, capture_output=True)
            with open(os.path.join(tmp, name + ".grid"), "rb") as f:
                gold["generator_kat"]["shapes/" + name] = hashlib.sha256(f.read()).hexdigest()
    with open(path, "w") as f:
        json.dump(gold, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main()
