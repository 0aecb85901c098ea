#!/bin/bash
# The reference's cubic-code pipeline with the decoder stage replaced by
# sogrand_b200's cubic_decoder.  The other stages are the reference's own C
# programs, compiled from its sources (directory given as $1, default the
# SOGRAND_C directory of a reference checkout) into a scratch directory.
#   usage: cubic_flow.sh <reference SOGRAND_C dir> [Eb/N0 dB]
set -euo pipefail
REFC=${1:?usage: cubic_flow.sh <reference SOGRAND_C dir> [Eb/N0 dB]}
SNR_DB=${2:-2.0}
HERE=$(cd "$(dirname "$0")/.." && pwd)
DECODER="$HERE/bin/cubic_decoder"
WORK=$(mktemp -d)
trap 'rm -rf "$WORK"' EXIT
cd "$WORK"
for stage in generate_bin cubic_encoder channel_sim comparator; do
    gcc "$REFC/$stage.c" -o "$stage" -lm
done
./generate_bin
./cubic_encoder original_data.bin encoded_cubic.bin
./channel_sim encoded_cubic.bin corrupted_llrs_cubic.bin "$SNR_DB" 3
"$DECODER" corrupted_llrs_cubic.bin decoded_cubic.bin
./comparator original_data.bin decoded_cubic.bin
