/*
 * Oracle harness I/O (test infrastructure only; never linked into the product).
 *
 * Shared by the harnesses that drive the reference's own Airfoil loops:
 *   ref_airfoil_seq.cpp  (reference op_seq.h, 8-argument update)
 *   ref_airfoil_gen.cpp  (input of the reference v1 translator: genseq/OpenMP)
 * Reads the binary mesh layout written by op2b.mesh.write_grid_bin (the same
 * arrays the reference driver reads from new_grid.dat,
 * apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:94-141) and writes the run's
 * results as raw little-endian arrays.
 */
#ifndef OP2B_REF_HARNESS_IO_H
#define OP2B_REF_HARNESS_IO_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int nnode, ncell, nedge, nbedge;
  double *x;
  int *cell, *edge, *ecell, *bedge, *becell, *bound;
} harness_mesh;

static void harness_die(const char *msg, const char *arg) {
  fprintf(stderr, "harness: %s %s\n", msg, arg ? arg : "");
  exit(2);
}

static void harness_read(FILE *f, void *dst, size_t bytes, const char *what) {
  if (bytes && fread(dst, 1, bytes, f) != bytes)
    harness_die("short read of", what);
}

static harness_mesh harness_read_mesh(const char *path) {
  harness_mesh m;
  int hdr[5];
  FILE *f = fopen(path, "rb");
  if (!f)
    harness_die("cannot open mesh", path);
  harness_read(f, hdr, sizeof(hdr), "header");
  if (hdr[0] != 0x4F503242)
    harness_die("bad magic in", path);
  m.nnode = hdr[1];
  m.ncell = hdr[2];
  m.nedge = hdr[3];
  m.nbedge = hdr[4];
  m.x = (double *)malloc(sizeof(double) * 2 * (size_t)m.nnode + 8);
  m.cell = (int *)malloc(sizeof(int) * 4 * (size_t)m.ncell + 8);
  m.edge = (int *)malloc(sizeof(int) * 2 * (size_t)m.nedge + 8);
  m.ecell = (int *)malloc(sizeof(int) * 2 * (size_t)m.nedge + 8);
  m.bedge = (int *)malloc(sizeof(int) * 2 * (size_t)m.nbedge + 8);
  m.becell = (int *)malloc(sizeof(int) * (size_t)m.nbedge + 8);
  m.bound = (int *)malloc(sizeof(int) * (size_t)m.nbedge + 8);
  harness_read(f, m.x, sizeof(double) * 2 * (size_t)m.nnode, "x");
  harness_read(f, m.cell, sizeof(int) * 4 * (size_t)m.ncell, "cell");
  harness_read(f, m.edge, sizeof(int) * 2 * (size_t)m.nedge, "edge");
  harness_read(f, m.ecell, sizeof(int) * 2 * (size_t)m.nedge, "ecell");
  harness_read(f, m.bedge, sizeof(int) * 2 * (size_t)m.nbedge, "bedge");
  harness_read(f, m.becell, sizeof(int) * (size_t)m.nbedge, "becell");
  harness_read(f, m.bound, sizeof(int) * (size_t)m.nbedge, "bound");
  fclose(f);
  return m;
}

static void harness_write(const char *prefix, const char *suffix,
                          const void *src, size_t bytes) {
  char path[4096];
  snprintf(path, sizeof(path), "%s.%s", prefix, suffix);
  FILE *f = fopen(path, "wb");
  if (!f)
    harness_die("cannot write", path);
  if (bytes && fwrite(src, 1, bytes, f) != bytes)
    harness_die("short write to", path);
  fclose(f);
}

#endif
