#!/usr/bin/env bash
# Run the reference Doki's own test scripts, unchanged, against a `doki`
# module: the reference's CI command list (pyproject.toml:28-44), plus one
# join_regs_tests range with cases in it (`-n 5` alone runs range(5, 5), no
# joins).  The scripts import `doki` by name, so PYTHONPATH selects the
# module under test.
#
#   tests/reference_scripts.sh <reference tests dir> [module dir]
#
# module dir: doki_b200 (this engine, needs a GPU; the default) or
# oracle/_ref (the reference compiled from its sources by oracle/Makefile).
# Exit status 0 when every command passes.
set -u
here="$(cd "$(dirname "$0")/.." && pwd)"
tests_dir="${1:?reference tests directory}"
module_dir="${2:-$here/doki_b200}"
fail=0
while read -r cmd; do
	[ -z "$cmd" ] && continue
	log="$(mktemp)"
	# shellcheck disable=SC2086
	if (cd "$tests_dir" && PYTHONPATH="$module_dir" timeout 600 python $cmd) > "$log" 2>&1; then
		echo "PASS $cmd"
	else
		echo "FAIL $cmd"
		tail -n 5 "$log"
		fail=1
	fi
	rm -f "$log"
done <<'LIST'
reg_creation_tests.py -n 1 -m 5
one_gate_tests.py -n 1 -m 5 -t 1
one_gate_tests.py -n 1 -m 5 -t 8
measure_tests.py -n 1 -m 5 -i 1000 -t 1
measure_tests.py -n 1 -m 5 -i 1000 -t 8
multiple_gate_tests.py -n 2 -m 5 -t 1
multiple_gate_tests.py -n 2 -m 5 -t 8
join_regs_tests.py -n 5 -t 1
join_regs_tests.py -n 5 -t 8
canonical_form_tests.py -n 1 -m 5
probability_tests.py -n 1 -m 5 -t 1
probability_tests.py -n 1 -m 5 -t 8
density_matrix_tests.py -n 1 -m 5
timed_test.py -n 5 -m 20 -t 1
timed_test.py -n 5 -m 20 -t 8
join_regs_tests.py -n 2 -m 5 -t 1
LIST
exit $fail
