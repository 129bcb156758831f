/*
 * vtk.c -- VTK XML output of one structured hex8 RVE: the .pvtu index and
 * its single piece _0.vtu, with the arrays the reference writes
 * (micro/src/output.c:65-188): point "displ" and "residual" (3 components),
 * cell "part", "strain", "stress" (6 Voigt components) and "elem_type".
 * Hexahedra are VTK cell type 12, connectivity in the hexa8 node order of
 * src/fem.c:324-362.  Floating-point data is written with %.9e (the
 * reference prints strain and stress with %lf, which keeps only six
 * decimals).
 */
#include <stdio.h>
#include <string.h>

#include "sp_internal.h"

static void elem_nodes(const int *n, int e, int *nod) {
  int nx = n[0] + 1, ny = n[1] + 1;
  int ex = e % n[0], ey = (e / n[0]) % n[1], ez = e / (n[0] * n[1]);
  int n0 = ex + ey * nx + ez * nx * ny;
  nod[0] = n0;
  nod[1] = n0 + 1;
  nod[2] = n0 + nx + 1;
  nod[3] = n0 + nx;
  for (int a = 0; a < 4; a++) nod[4 + a] = nod[a] + nx * ny;
}

int sp_vtu_write(const char *base, const int *n, const double *len, const double *u,
                 const double *res, const unsigned char *etype, const double *strain_e,
                 const double *stress_e) {
  if (!base || !n || !len) return sp_set_error(SP_ERR_ARG, "sp_vtu_write: null argument");
  for (int k = 0; k < 3; k++)
    if (n[k] < 1 || !(len[k] > 0)) return sp_set_error(SP_ERR_ARG, "sp_vtu_write: bad mesh");
  if (strlen(base) > 1000) return sp_set_error(SP_ERR_ARG, "sp_vtu_write: path too long");
  const int nx = n[0] + 1, ny = n[1] + 1, nz = n[2] + 1;
  const int nn = nx * ny * nz, nelm = n[0] * n[1] * n[2];
  const double h[3] = {len[0] / n[0], len[1] / n[1], len[2] / n[2]};
  char path[1100];
  const char *leaf = strrchr(base, '/');
  leaf = leaf ? leaf + 1 : base;

  snprintf(path, sizeof(path), "%s.pvtu", base);
  FILE *f = fopen(path, "w");
  if (!f) return sp_set_error(SP_ERR_ARG, "sp_vtu_write: cannot open %s", path);
  fprintf(f,
          "<?xml version=\"1.0\"?>\n"
          "<VTKFile type=\"PUnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
          "<PUnstructuredGrid GhostLevel=\"0\">\n"
          "<PPoints>\n"
          "<PDataArray type=\"Float32\" Name=\"Position\" NumberOfComponents=\"3\"/>\n"
          "</PPoints>\n"
          "<PCells>\n"
          "<PDataArray type=\"Int32\" Name=\"connectivity\" NumberOfComponents=\"1\"/>\n"
          "<PDataArray type=\"Int32\" Name=\"offsets\" NumberOfComponents=\"1\"/>\n"
          "<PDataArray type=\"UInt8\" Name=\"types\" NumberOfComponents=\"1\"/>\n"
          "</PCells>\n"
          "<PPointData Vectors=\"displ\">\n"
          "<PDataArray type=\"Float64\" Name=\"displ\" NumberOfComponents=\"3\"/>\n"
          "<PDataArray type=\"Float64\" Name=\"residual\" NumberOfComponents=\"3\"/>\n"
          "</PPointData>\n"
          "<PCellData>\n"
          "<PDataArray type=\"Int32\" Name=\"part\" NumberOfComponents=\"1\"/>\n"
          "<PDataArray type=\"Float64\" Name=\"strain\" NumberOfComponents=\"6\"/>\n"
          "<PDataArray type=\"Float64\" Name=\"stress\" NumberOfComponents=\"6\"/>\n"
          "<PDataArray type=\"Int32\" Name=\"elem_type\" NumberOfComponents=\"1\"/>\n"
          "</PCellData>\n"
          "<Piece Source=\"%s_0.vtu\"/>\n"
          "</PUnstructuredGrid>\n</VTKFile>\n",
          leaf);
  if (fclose(f)) return sp_set_error(SP_ERR_ARG, "sp_vtu_write: write failed");

  snprintf(path, sizeof(path), "%s_0.vtu", base);
  f = fopen(path, "w");
  if (!f) return sp_set_error(SP_ERR_ARG, "sp_vtu_write: cannot open %s", path);
  fprintf(f,
          "<?xml version=\"1.0\"?>\n"
          "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
          "<UnstructuredGrid>\n"
          "<Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n"
          "<Points>\n"
          "<DataArray type=\"Float32\" Name=\"Position\" NumberOfComponents=\"3\" format=\"ascii\">\n",
          nn, nelm);
  for (int a = 0; a < nn; a++) {
    int i = a % nx, j = (a / nx) % ny, k = a / (nx * ny);
    fprintf(f, "%e %e %e\n", i * h[0], j * h[1], k * h[2]);
  }
  fprintf(f, "</DataArray>\n</Points>\n<Cells>\n"
             "<DataArray type=\"Int32\" Name=\"connectivity\" NumberOfComponents=\"1\" format=\"ascii\">\n");
  for (int e = 0; e < nelm; e++) {
    int nod[8];
    elem_nodes(n, e, nod);
    for (int a = 0; a < 8; a++) fprintf(f, "%d%s", nod[a], a == 7 ? "\n" : " ");
  }
  fprintf(f, "</DataArray>\n"
             "<DataArray type=\"Int32\" Name=\"offsets\" NumberOfComponents=\"1\" format=\"ascii\">\n");
  for (int e = 0; e < nelm; e++) fprintf(f, "%d ", 8 * (e + 1));
  fprintf(f, "\n</DataArray>\n"
             "<DataArray type=\"UInt8\" Name=\"types\" NumberOfComponents=\"1\" format=\"ascii\">\n");
  for (int e = 0; e < nelm; e++) fprintf(f, "12 ");
  fprintf(f, "\n</DataArray>\n</Cells>\n<PointData Vectors=\"displ\">\n");
  const double *pv[2] = {u, res};
  const char *pn[2] = {"displ", "residual"};
  for (int v = 0; v < 2; v++) {
    fprintf(f, "<DataArray type=\"Float64\" Name=\"%s\" NumberOfComponents=\"3\" format=\"ascii\">\n",
            pn[v]);
    for (int a = 0; a < nn; a++)
      for (int d = 0; d < 3; d++)
        fprintf(f, "%.9e%s", pv[v] ? pv[v][3 * a + d] : 0.0, d == 2 ? "\n" : " ");
    fprintf(f, "</DataArray>\n");
  }
  fprintf(f, "</PointData>\n<CellData>\n"
             "<DataArray type=\"Int32\" Name=\"part\" NumberOfComponents=\"1\" format=\"ascii\">\n");
  for (int e = 0; e < nelm; e++) fprintf(f, "0 ");
  fprintf(f, "\n</DataArray>\n");
  const double *cv[2] = {strain_e, stress_e};
  const char *cn[2] = {"strain", "stress"};
  for (int v = 0; v < 2; v++) {
    fprintf(f, "<DataArray type=\"Float64\" Name=\"%s\" NumberOfComponents=\"6\" format=\"ascii\">\n",
            cn[v]);
    for (int e = 0; e < nelm; e++)
      for (int c = 0; c < 6; c++)
        fprintf(f, "%.9e%s", cv[v] ? cv[v][6 * e + c] : 0.0, c == 5 ? "\n" : " ");
    fprintf(f, "</DataArray>\n");
  }
  fprintf(f, "<DataArray type=\"Int32\" Name=\"elem_type\" NumberOfComponents=\"1\" format=\"ascii\">\n");
  for (int e = 0; e < nelm; e++) fprintf(f, "%d ", etype ? (int)etype[e] : 0);
  fprintf(f, "\n</DataArray>\n</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
  if (fclose(f)) return sp_set_error(SP_ERR_ARG, "sp_vtu_write: write failed");
  return SP_OK;
}
