"""Copies the reference's golden run fixture into tests/golden/run_tiny/ (run once, in a container
that has the reference checked out; the copies are committed so the tests need no reference).

The fixture is the run `write_tiny` in crates/waveio/tests/golden.rs:18-78 writes, which the
reference compares byte for byte (golden.rs:80-104) and its viewer's tests read:
viewer/tests/fixtures/tiny/{run.json, bed.f32, frames.f32}.

    python tests/golden/copy_reference_fixtures.py [reference root]
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    src = os.path.join(root, "viewer", "tests", "fixtures", "tiny")
    dst = os.path.join(HERE, "run_tiny")
    os.makedirs(dst, exist_ok=True)
    for name in ("run.json", "bed.f32", "frames.f32"):
        shutil.copyfile(os.path.join(src, name), os.path.join(dst, name))
        print(name, os.path.getsize(os.path.join(dst, name)), "bytes")


if __name__ == "__main__":
    main()
