"""The gate-fusion planner (doki_b200/csrc/dk_plan.c, host C) under
AddressSanitizer and UndefinedBehaviorSanitizer, on CPU.

A C driver builds plans for seeded random circuits -- 3 to 30 qubits, gates
on 1 to 5 qubits of every kind the planner classifies (dense, diagonal,
anti-diagonal, phase, sign flip, swap), controls and anticontrols inside and
outside the tile, brickwork layers like the benchmark circuit -- under every
planner option (tensor and scalar sweeps, tile widths, pinned low qubits,
folding, fusion off), walks each plan's steps and sweep headers, and frees
it.  Any out-of-bounds access, use after free, leak or undefined operation
aborts the driver.
"""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

from tests.conftest import ROOT

DRIVER = r"""
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "dk_internal.h"

static uint64_t rs = 88172645463325252ull;
static uint64_t rnd(void)
{
	rs ^= rs << 13;
	rs ^= rs >> 7;
	rs ^= rs << 17;
	return rs;
}
static unsigned below(unsigned n) { return (unsigned)(rnd() % n); }
static double unit(void) { return (double)(rnd() >> 11) / 9007199254740992.0 - 0.5; }
/* a qubit is still free for another control */
static int popcount_free(uint64_t taken, unsigned n)
{
	return (unsigned)__builtin_popcountll(taken) < n;
}

/* a gate of one of the planner's kinds on k qubits */
static struct dk_gate *make_gate(unsigned k)
{
	struct dk_gate *g = calloc(1, sizeof(*g));
	g->k = k;
	g->dim = 1ull << k;
	g->m = calloc(2 * g->dim * g->dim, sizeof(double));
	const unsigned kind = below(6);
	for (uint64_t r = 0; r < g->dim; r++)
		for (uint64_t c = 0; c < g->dim; c++) {
			double *e = g->m + 2 * (r * g->dim + c);
			int on;
			switch (kind) {
			case 0: on = 1; break;                             /* dense */
			case 1: on = (r == c); break;                      /* diagonal */
			case 2: on = (r ^ c) == g->dim - 1; break;         /* anti-diagonal */
			default: on = (r == c); break;
			}
			if (!on)
				continue;
			if (kind == 3) { /* phase: 1 ... e^{i t} */
				e[0] = (r + 1 == g->dim) ? 0.6 : 1.0;
				e[1] = (r + 1 == g->dim) ? 0.8 : 0.0;
			} else if (kind == 4) { /* sign flip */
				e[0] = (r + 1 == g->dim) ? -1.0 : 1.0;
			} else if (kind == 5 && k == 1) { /* X */
				e[0] = 0.0;
				g->m[2 * (r * 2 + (1 - r))] = 1.0;
			} else {
				e[0] = unit();
				e[1] = unit();
			}
		}
	return g;
}

static void free_gate(struct dk_gate *g)
{
	free(g->m);
	free(g);
}

static int check_plan(const dk_plan *p, int nops)
{
	for (int i = 0; i < p->nsteps; i++) {
		const dk_step *s = &p->steps[i];
		if (s->kind == 2) {
			if (s->op_index < 0 || s->op_index >= nops)
				return 1;
		} else if (s->kind == 1) {
			if (s->prog_off + sizeof(dk_sweep_hdr) > p->blob_bytes)
				return 2;
			const dk_sweep_hdr *h = (const dk_sweep_hdr *)(p->blob + s->prog_off);
			if (s->prog_off + h->bytes > p->blob_bytes || h->npass <= 0)
				return 3;
		} else {
			return 4;
		}
	}
	return 0;
}

int main(int argc, char **argv)
{
	const int trials = argc > 1 ? atoi(argv[1]) : 300;
	for (int t = 0; t < trials; t++) {
		const unsigned n = 3 + below(28);
		const int brick = (t % 4) == 0;
		int nops = brick ? 0 : 1 + (int)below(200);
		const int layers = brick ? 2 + (int)below(6) : 0;
		if (brick)
			nops = layers * (int)(n + n / 2);
		dk_flat_op *ops = calloc((size_t)nops, sizeof(dk_flat_op));
		struct dk_gate **gates = calloc((size_t)nops, sizeof(*gates));
		int used = 0;
		for (int l = 0; brick && l < layers; l++) {
			for (unsigned q = 0; q < n; q++) {
				gates[used] = make_gate(1);
				ops[used].gate = gates[used];
				ops[used].k = 1;
				ops[used].tg[0] = q;
				used++;
			}
			for (unsigned a = (unsigned)l % 2; a + 1 < n; a += 2) {
				gates[used] = make_gate(1);
				ops[used].gate = gates[used];
				ops[used].k = 1;
				ops[used].tg[0] = a;
				ops[used].cm = 1ull << (a + 1);
				if (below(20) == 0)
					ops[used].am = 1ull << ((a + 2 + below(n - 2)) % n) & ~(3ull << a);
				used++;
			}
		}
		for (; !brick && used < nops; used++) {
			unsigned k = 1 + below(3);
			if (below(25) == 0)
				k = 4 + below(2);
			if (k > n)
				k = n;
			gates[used] = make_gate(k);
			ops[used].gate = gates[used];
			ops[used].k = k;
			uint64_t taken = 0;
			for (unsigned j = 0; j < k; j++) {
				unsigned q;
				do
					q = below(n);
				while (taken >> q & 1u);
				taken |= 1ull << q;
				ops[used].tg[j] = q;
			}
			const unsigned nc = below(4);
			for (unsigned j = 0; j < nc && popcount_free(taken, n); j++) {
				unsigned q;
				do
					q = below(n);
				while (taken >> q & 1u);
				taken |= 1ull << q;
				if (below(2))
					ops[used].cm |= 1ull << q;
				else
					ops[used].am |= 1ull << q;
			}
		}
		nops = used;
		dk_plan_limits lim;
		memset(&lim, 0, sizeof(lim));
		lim.tensor = below(2) ? 0 : -1;
		lim.fold = (int[]){ -1, 0, 1, 400 }[below(4)];
		lim.tile_bits = below(3) ? 0 : 6 + (int)below(7);
		const int prec = below(2) ? DK_C128 : DK_C64;
		dk_plan_default_limits(prec, n, &lim);
		if (below(3) == 0)
			lim.low_bits = (int)below((unsigned)lim.tile_bits + 1);
		if (below(8) == 0)
			lim.fuse = 0;
		dk_plan plan;
		memset(&plan, 0, sizeof(plan));
		const int rc = dk_plan_build(ops, nops, n, prec, &lim, &plan);
		if (rc != 0) {
			fprintf(stderr, "trial %d: dk_plan_build returned %d\n", t, rc);
			return 10;
		}
		const int bad = check_plan(&plan, nops);
		if (bad) {
			fprintf(stderr, "trial %d: malformed plan (%d)\n", t, bad);
			return 11;
		}
		dk_plan_free(&plan);
		for (int i = 0; i < nops; i++)
			free_gate(gates[i]);
		free(gates);
		free(ops);
	}
	printf("ok %d\n", trials);
	return 0;
}
"""


def test_planner_under_asan_and_ubsan(tmp_path):
    gcc = shutil.which("gcc") or "/usr/bin/gcc"
    csrc = os.path.join(ROOT, "doki_b200", "csrc")
    drv = tmp_path / "plan_driver.c"
    drv.write_text(DRIVER)
    exe = tmp_path / "plan_asan"
    cmd = [gcc, "-std=gnu11", "-O1", "-g", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=all", "-fno-omit-frame-pointer",
           "-I", os.path.join(ROOT, "include"), "-I", csrc,
           os.path.join(csrc, "dk_plan.c"), str(drv), "-lm", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 and "asan" in r.stderr.lower():
        pytest.skip("sanitizer runtime unavailable: " + r.stderr[-200:])
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1")
    run = subprocess.run([str(exe), "400"], capture_output=True, text=True, env=env,
                         timeout=600)
    if run.returncode != 0 and "LeakSanitizer has encountered a fatal error" in run.stderr:
        env["ASAN_OPTIONS"] = "detect_leaks=0"
        run = subprocess.run([str(exe), "400"], capture_output=True, text=True, env=env,
                             timeout=600)
    assert run.returncode == 0, run.stderr[-3000:]
    assert run.stdout.strip() == "ok 400"
