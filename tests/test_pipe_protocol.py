"""The warp kernel's pipelined launch (csrc/gcl_capi.cu, w64_pipe_kernel):
its root claims, inline searches and search-slot queue run by host threads
with C11 atomics.  Each thread plays a warp: it claims graphs from a counter
and does each one's root step; a graph finished at its root is done there, a
costly one is searched by the same thread at once (counted as rooted first),
any other is written to the next root slot and flagged ready.  With no graph
left to claim, a thread takes a ticket of the queue, waits until the ticket's
slot exists (or every root is done and the ticket is past the last slot),
waits for the slot's flag and searches that graph.  Checked under real
interleavings with random work sizes: every graph is finished exactly once --
at its root, inline or from its slot -- no wait runs out, and every thread
stops.  CPU only."""
import os
import subprocess

import pytest

SRC = r'''
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#define MAXG 20000
#define WAIT (1ul << 30)
static atomic_int next_graph, search_count, next_search, roots_done, timeouts;
static atomic_int ready[MAXG];
static int slot_graph[MAXG];
static atomic_int finished[MAXG];
static int kind[MAXG], cost[MAXG];  /* 0 discrete root, 1 searched inline, 2 queued */
static int count;

static void spin(int units, unsigned* seed) {
  volatile unsigned x = *seed;
  for (int i = 0; i < units; ++i) x = x * 1103515245u + 12345u;
  *seed = x;
}

static void* warp(void* arg) {
  unsigned seed = (unsigned)(uintptr_t)arg;
  for (;;) {  /* roots */
    const int i = atomic_fetch_add(&next_graph, 1);
    if (i >= count) break;
    spin(50 + cost[i] % 200, &seed);  /* the root refinement */
    if (kind[i] == 1) {
      atomic_fetch_add(&roots_done, 1);
      spin(cost[i], &seed);           /* the search, at once */
      atomic_fetch_add(&finished[i], 1);
      continue;
    }
    if (kind[i] == 2) {
      const int j = atomic_fetch_add(&search_count, 1);
      slot_graph[j] = i;              /* the root slot */
      atomic_thread_fence(memory_order_seq_cst);
      atomic_store(&ready[j], 1);
    } else {
      atomic_fetch_add(&finished[i], 1);
    }
    atomic_thread_fence(memory_order_seq_cst);
    atomic_fetch_add(&roots_done, 1);
  }
  for (;;) {  /* the search queue */
    const int t = atomic_fetch_add(&next_search, 1);
    int ok = 0;
    unsigned long it = 0;
    for (; it < WAIT; ++it) {
      if (atomic_load(&search_count) > t) { ok = 1; break; }
      if (atomic_load(&roots_done) >= count) {
        atomic_thread_fence(memory_order_seq_cst);
        ok = atomic_load(&search_count) > t;
        break;
      }
    }
    if (it == WAIT) atomic_fetch_add(&timeouts, 1);
    if (ok) {
      unsigned long k = 0;
      while (!atomic_load(&ready[t]) && k < WAIT) ++k;
      if (k == WAIT) { atomic_fetch_add(&timeouts, 1); ok = 0; }
      atomic_thread_fence(memory_order_seq_cst);
    }
    if (!ok) return NULL;
    const int g = slot_graph[t];
    spin(cost[g], &seed);
    atomic_fetch_add(&finished[g], 1);
  }
}

int main(int argc, char** argv) {
  const int threads = atoi(argv[1]);
  unsigned seed = (unsigned)atoi(argv[2]);
  count = 1 + (int)(seed % 3000);
  int queued = 0, inline_ = 0;
  for (int g = 0; g < count; ++g) {
    seed = seed * 1103515245u + 12345u;
    const unsigned r = (seed >> 8) % 100;
    kind[g] = r < 23 ? 0 : (r < 25 ? 1 : 2);
    cost[g] = kind[g] == 1 ? 20000 + (int)(seed % 20000) : (int)(seed % 3000);
    queued += kind[g] == 2;
    inline_ += kind[g] == 1;
  }
  pthread_t th[64];
  for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, warp, (void*)(uintptr_t)(t + 1));
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  int bad = 0;
  for (int g = 0; g < count; ++g) bad += atomic_load(&finished[g]) != 1;
  printf("%d %d %d %d %d\n", bad, atomic_load(&timeouts), atomic_load(&search_count), queued,
         inline_);
  return 0;
}
'''


@pytest.fixture(scope="module")
def proto(tmp_path_factory):
    d = tmp_path_factory.mktemp("pipe")
    (d / "p.c").write_text(SRC)
    exe = d / "p"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-O2", "-std=c11", "-pthread", "-o", str(exe), str(d / "p.c")], check=True)
    return exe


def test_every_graph_finished_once_and_every_thread_stops(proto):
    queued_total = inline_total = 0
    for threads in (1, 2, 7, 16, 48):
        for seed in range(1, 7):
            r = subprocess.run([str(proto), str(threads), str(seed * 131 + threads)],
                               capture_output=True, text=True, timeout=120)
            assert r.returncode == 0, r.stderr
            bad, timeouts, slots, queued, inline_ = map(int, r.stdout.split())
            assert bad == 0 and timeouts == 0, (threads, seed)
            assert slots == queued  # every queued graph got exactly one slot
            queued_total += queued
            inline_total += inline_
    assert queued_total > 0 and inline_total > 0  # both paths taken
