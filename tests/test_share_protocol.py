"""The wide search's work-sharing protocol (csrc/canon_wide.cuh:
wide_try_donate, wide_take_gift and the busy count around each item) run by
host threads with C11 atomics: every unit of work is done exactly once and
every thread stops, under real interleavings.  Each thread plays a warp: it
takes items from a counter, hands half of its remaining work to the queue
while threads are waiting, and when the items are gone waits for handed-over
work until no thread is busy and the queue is empty -- reading the busy count
before the queue, as the kernel does.  CPU only."""
import os
import subprocess

import pytest

SRC = r'''
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#define QCAP 4096
static atomic_uint next_item, busy, hungry, qhead, qtail, ready[QCAP];
static atomic_ulong done_units;
static unsigned work[QCAP];
static unsigned nitems, item_work[4096];

static void process(unsigned units, unsigned seed) {
  while (units > 0) {
    atomic_fetch_add(&done_units, 1);
    --units;
    seed = seed * 1103515245u + 12345u;
    if ((seed >> 16) % 4 == 0 && units > 1) {      /* wide_try_donate */
      unsigned h = atomic_load(&hungry), hd = atomic_load(&qhead), tl = atomic_load(&qtail);
      if (h > tl - hd && tl < QCAP) {
        for (int tries = 0; tries < 64; ++tries) {
          unsigned t = atomic_load(&qtail);
          if (t >= QCAP) break;
          if (atomic_compare_exchange_strong(&qtail, &t, t + 1)) {
            unsigned give = units / 2;
            work[t] = give;
            units -= give;
            atomic_store(&ready[t], 1);
            break;
          }
        }
      }
    }
  }
}

static void* warp(void* arg) {
  unsigned seed = (unsigned)(uintptr_t)arg;
  for (;;) {
    unsigned it = atomic_fetch_add(&next_item, 1);
    if (it < nitems) {
      atomic_fetch_add(&busy, 1);
      process(item_work[it], seed ^ it);
      atomic_thread_fence(memory_order_seq_cst);
      atomic_fetch_sub(&busy, 1);
      continue;
    }
    /* wide_take_gift */
    atomic_fetch_add(&hungry, 1);
    unsigned got = ~0u;
    for (unsigned long i = 0;; ++i) {
      unsigned b = atomic_load(&busy);
      atomic_thread_fence(memory_order_seq_cst);
      unsigned hd = atomic_load(&qhead), tl = atomic_load(&qtail);
      if (hd < tl) {
        if (atomic_compare_exchange_strong(&qhead, &hd, hd + 1)) { got = hd; break; }
        continue;
      }
      if (b == 0) break;
      if (i > 200000000ul) { fprintf(stderr, "stuck\n"); exit(3); }
    }
    if (got == ~0u) { atomic_fetch_sub(&hungry, 1); return NULL; }
    atomic_fetch_add(&busy, 1);
    while (!atomic_load(&ready[got])) {}
    atomic_fetch_sub(&hungry, 1);
    process(work[got], seed ^ (got * 7919u));
    atomic_thread_fence(memory_order_seq_cst);
    atomic_fetch_sub(&busy, 1);
  }
}

int main(int argc, char** argv) {
  int threads = atoi(argv[1]);
  unsigned seed = (unsigned)atoi(argv[2]);
  unsigned long total = 0;
  nitems = 1 + seed % 40;
  for (unsigned i = 0; i < nitems; ++i) {
    seed = seed * 1103515245u + 12345u;
    item_work[i] = (seed >> 8) % (i == 0 ? 20000 : 200);  /* one heavy item */
    total += item_work[i];
  }
  pthread_t th[64];
  for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, warp, (void*)(uintptr_t)(t + 1));
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  printf("%lu %lu %u\n", (unsigned long)atomic_load(&done_units), total, atomic_load(&qtail));
  return 0;
}
'''


@pytest.fixture(scope="module")
def proto(tmp_path_factory):
    d = tmp_path_factory.mktemp("share")
    (d / "p.c").write_text(SRC)
    exe = d / "p"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-O2", "-std=c11", "-pthread", "-o", str(exe), str(d / "p.c")], check=True)
    return exe


def test_every_unit_once_and_every_thread_stops(proto):
    handed = 0
    for threads in (2, 5, 16, 48):
        for seed in range(1, 9):
            r = subprocess.run([str(proto), str(threads), str(seed * 97 + threads)],
                               capture_output=True, text=True, timeout=120)
            assert r.returncode == 0, r.stderr
            done, total, queued = map(int, r.stdout.split())
            assert done == total, (threads, seed)
            handed += queued
    assert handed > 0  # work was actually handed over
