// ref_plan_dump.cpp -- calls the reference's own op_plan_core
// (common/op_lib_core.c:627-1089, compiled unmodified by oracle/Makefile)
// on a loop described in a text spec and writes every plan array as raw
// int32 / int16 files.  TEST INFRASTRUCTURE ONLY: it produces golden plans.
//
// spec (whitespace separated):
//   name loop_set part_size nargs ninds nsets nmaps
//   nsets x  : set_size
//   nmaps x  : from_set to_set dim path_to_int32_file
//   nargs x  : map(-1 = OP_ID) idx dat_dim dat_elem_bytes acc ind dat_id
// Args with the same dat_id share one op_dat (like the apps' p_x, p_q ...).

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "op_lib.h"

int OP2REF_dummy;

static void write_raw(const std::string &dir, const char *name, const void *p, size_t bytes) {
  std::string path = dir + "/" + name;
  FILE *fp = fopen(path.c_str(), "wb");
  if (!fp) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(1); }
  if (bytes) fwrite(p, 1, bytes, fp);
  fclose(fp);
}

int main(int argc, char **argv) {
  if (argc < 3) { fprintf(stderr, "usage: %s spec outdir\n", argv[0]); return 2; }
  FILE *fp = fopen(argv[1], "r");
  if (!fp) { fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
  std::string out = argv[2];

  char name[256];
  int loop_id, part_size, nargs, ninds, nsets, nmaps;
  if (fscanf(fp, "%255s %d %d %d %d %d %d", name, &loop_id, &part_size, &nargs, &ninds,
             &nsets, &nmaps) != 7) return 3;

  op_init_core(0, NULL, 0);

  std::vector<op_set> sets(nsets);
  for (int s = 0; s < nsets; s++) {
    int sz;
    if (fscanf(fp, "%d", &sz) != 1) return 3;
    sets[s] = op_decl_set(sz, "s");
  }
  std::vector<op_map> maps(nmaps);
  for (int k = 0; k < nmaps; k++) {
    int from, to, dim;
    char path[4096];
    if (fscanf(fp, "%d %d %d %4095s", &from, &to, &dim, path) != 4) return 3;
    size_t n = (size_t)sets[from]->size * dim;
    int *data = (int *)malloc(n * sizeof(int));
    FILE *mf = fopen(path, "rb");
    if (!mf || fread(data, sizeof(int), n, mf) != n) { fprintf(stderr, "bad map %s\n", path); return 3; }
    fclose(mf);
    maps[k] = op_decl_map(sets[from], sets[to], dim, data, "m");
  }

  std::vector<op_arg> args(nargs);
  std::vector<int> inds(nargs);
  std::vector<op_dat> dats(64, (op_dat)NULL);
  op_set loop_set = sets[loop_id];
  for (int m = 0; m < nargs; m++) {
    int map, idx, dim, bytes, acc, ind, dat_id;
    if (fscanf(fp, "%d %d %d %d %d %d %d", &map, &idx, &dim, &bytes, &acc, &ind, &dat_id) != 7)
      return 3;
    op_set dset = map >= 0 ? maps[map]->to : loop_set;
    if (!dats[dat_id])
      dats[dat_id] = op_decl_dat_core(dset, dim, "float", bytes, (char *)&OP2REF_dummy, "d");
    args[m] = op_arg_dat(dats[dat_id], idx, map >= 0 ? maps[map] : NULL, dim, "float",
                         (op_access)acc);
    inds[m] = ind;
  }
  fclose(fp);

  op_plan *p = op_plan_core(name, loop_set, part_size, nargs, args.data(), ninds, inds.data());

  FILE *meta = fopen((out + "/meta.txt").c_str(), "w");
  fprintf(meta, "nblocks %d\nncolors %d\nnshared %d\ntransfer %.9g\ntransfer2 %.9g\n", p->nblocks,
          p->ncolors, p->nshared, p->transfer, p->transfer2);
  fclose(meta);
  int nb = p->nblocks, n = loop_set->size;
  write_raw(out, "nthrcol.i32", p->nthrcol, sizeof(int) * nb);
  write_raw(out, "thrcol.i32", p->thrcol, sizeof(int) * n);
  write_raw(out, "offset.i32", p->offset, sizeof(int) * nb);
  write_raw(out, "nelems.i32", p->nelems, sizeof(int) * nb);
  write_raw(out, "blkmap.i32", p->blkmap, sizeof(int) * nb);
  write_raw(out, "ncolblk.i32", p->ncolblk, sizeof(int) * p->ncolors);
  write_raw(out, "ind_offs.i32", p->ind_offs, sizeof(int) * nb * ninds);
  write_raw(out, "ind_sizes.i32", p->ind_sizes, sizeof(int) * nb * ninds);
  write_raw(out, "nindirect.i32", p->nindirect, sizeof(int) * ninds);
  char fn[64];
  for (int m = 0; m < ninds; m++) {
    snprintf(fn, sizeof fn, "ind_maps%d.i32", m);
    write_raw(out, fn, p->ind_maps[m], sizeof(int) * p->nindirect[m]);
  }
  for (int m = 0; m < nargs; m++)
    if (p->loc_maps[m]) {
      snprintf(fn, sizeof fn, "loc_maps%d.i16", m);
      write_raw(out, fn, p->loc_maps[m], sizeof(short) * n);
    }
  return 0;
}
