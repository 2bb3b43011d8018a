#!/usr/bin/env bash
# Install the unmodified reference (proton_solver) for `bench.py --impl reference`.
#
#   baseline/install_reference.sh <reference root>
#
# The package goes to baseline/_ref/lib, and its coefficient tables to
# baseline/_ref/data: the package finds its tables three directories above its
# physics modules, which is baseline/_ref/data for this layout.  Only the four
# tables the energy march reads are copied (materials.csv, stopping_power,
# nuclear_attenuation, wentzel_transport; not the CT volumes), and
# baseline/synth_tables.py adds this library's synthetic materials to them.
#
# The install is offline (--no-index, the image's wheelhouse).  --no-deps: the
# reference pins matplotlib>=3.11.1, numba>=0.67 and numpy>=2.4.6, which the
# wheelhouse does not carry.  The energy march runs on the image's numba 0.65
# and numpy 2.3, and bench.py gives empty stand-ins for the plotting and
# gamma-index modules (matplotlib, pymedphys) that the package imports.
# baseline/_ref is git-ignored and travels with the working tree.
set -euo pipefail
src=${1:?usage: install_reference.sh <reference root>}
here=$(cd "$(dirname "$0")" && pwd)
tmp=$(mktemp -d)
trap 'rm -rf "$tmp"' EXIT
# the build writes into its source tree: build from a copy
cp -r "$src" "$tmp/src"
rm -rf "$here/_ref"
python -m pip install --no-index --no-build-isolation --no-deps \
    --find-links /opt/wheelhouse --target "$here/_ref/lib" "$tmp/src"
mkdir -p "$here/_ref/data"
for t in materials.csv stopping_power nuclear_attenuation wentzel_transport; do
    cp -r "$src/data/$t" "$here/_ref/data/"
done
# this library's synthetic materials (ADIPOSE_SYNTH), in the reference's table formats
python "$here/synth_tables.py" "$here/_ref/data"
echo "reference installed under $here/_ref"
