/*
 * output.c - VTK XML unstructured-grid files of uniform grids with cell
 * data, the format the reference writes through PETSc's VTU viewer every
 * outputfreq steps (src/cipher.c:1080-1089: "<outfile>_<step>.vtu").
 *
 * Layout of the file: the header names every array with an offset into one
 * raw appended-data block; each array there is a UInt64 byte count followed
 * by its little-endian values.  Points are the grid's nodes (x fastest),
 * cells are lines, quads or hexahedra in cell order, cell data are Float64.
 */
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>
#include "cipher_problem.h"
#include "cipher_b200.h"

static int write_block(FILE *f, const void *data, uint64_t nbytes)
{
    if (fwrite(&nbytes, sizeof(nbytes), 1, f) != 1) return -1;
    if (nbytes && fwrite(data, 1, (size_t)nbytes, f) != (size_t)nbytes) return -1;
    return 0;
}

int cipher_write_vtu(const char *path, const cipher_problem *p, const cipher_output_field *fields, int nfields,
                     const double *values)
{
    if (!path || !p || (nfields > 0 && (!fields || !values))) return CIPHER_E_ARG;
    const int dim = p->dim;
    int r[3] = {1, 1, 1};
    double h[3] = {1.0, 1.0, 1.0};
    for (int d = 0; d < dim; d++) {
        r[d] = p->resolution[d];
        h[d] = p->size[d] / r[d];
    }
    const int nr[3] = {r[0] + 1, dim > 1 ? r[1] + 1 : 1, dim > 2 ? r[2] + 1 : 1};
    const int64_t npts = (int64_t)nr[0] * nr[1] * nr[2];
    const int64_t ncells = (int64_t)r[0] * r[1] * r[2];
    const int nv = dim == 1 ? 2 : dim == 2 ? 4 : 8;
    const uint8_t vtype = dim == 1 ? 3 : dim == 2 ? 9 : 12;   /* VTK_LINE, VTK_QUAD, VTK_HEXAHEDRON */

    double *pts = (double *)malloc((size_t)npts * 3 * sizeof(double));
    int64_t *conn = (int64_t *)malloc((size_t)ncells * nv * sizeof(int64_t));
    int64_t *offs = (int64_t *)malloc((size_t)ncells * sizeof(int64_t));
    uint8_t *types = (uint8_t *)malloc((size_t)ncells);
    if (!pts || !conn || !offs || !types) { free(pts); free(conn); free(offs); free(types); return CIPHER_E_NOMEM; }
    for (int64_t k = 0; k < npts; k++) {
        const int64_t i = k % nr[0], j = (k / nr[0]) % nr[1], l = k / ((int64_t)nr[0] * nr[1]);
        pts[3 * k + 0] = i * h[0];
        pts[3 * k + 1] = dim > 1 ? j * h[1] : 0.0;
        pts[3 * k + 2] = dim > 2 ? l * h[2] : 0.0;
    }
#define NODE(i, j, l) ((int64_t)(i) + (int64_t)nr[0] * ((int64_t)(j) + (int64_t)nr[1] * (l)))
    for (int64_t c = 0; c < ncells; c++) {
        const int64_t i = c % r[0], j = (c / r[0]) % r[1], l = c / ((int64_t)r[0] * r[1]);
        int64_t *q = &conn[c * nv];
        if (dim == 1) {
            q[0] = NODE(i, 0, 0); q[1] = NODE(i + 1, 0, 0);
        } else if (dim == 2) {
            q[0] = NODE(i, j, 0); q[1] = NODE(i + 1, j, 0); q[2] = NODE(i + 1, j + 1, 0); q[3] = NODE(i, j + 1, 0);
        } else {
            q[0] = NODE(i, j, l); q[1] = NODE(i + 1, j, l); q[2] = NODE(i + 1, j + 1, l); q[3] = NODE(i, j + 1, l);
            q[4] = NODE(i, j, l + 1); q[5] = NODE(i + 1, j, l + 1); q[6] = NODE(i + 1, j + 1, l + 1); q[7] = NODE(i, j + 1, l + 1);
        }
        offs[c] = (c + 1) * nv;
        types[c] = vtype;
    }
#undef NODE
    FILE *f = fopen(path, "wb");
    if (!f) { free(pts); free(conn); free(offs); free(types); return CIPHER_E_ARG; }
    uint64_t off = 0;
    const uint64_t b_pts = (uint64_t)npts * 3 * 8, b_conn = (uint64_t)ncells * nv * 8, b_offs = (uint64_t)ncells * 8,
                   b_types = (uint64_t)ncells, b_field = (uint64_t)ncells * 8;
    fprintf(f, "<?xml version=\"1.0\"?>\n");
    fprintf(f, "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
    fprintf(f, "  <UnstructuredGrid>\n    <Piece NumberOfPoints=\"%lld\" NumberOfCells=\"%lld\">\n",
            (long long)npts, (long long)ncells);
    fprintf(f, "      <Points>\n        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"appended\" offset=\"%llu\"/>\n      </Points>\n",
            (unsigned long long)off);
    off += 8 + b_pts;
    fprintf(f, "      <Cells>\n");
    fprintf(f, "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"appended\" offset=\"%llu\"/>\n", (unsigned long long)off);
    off += 8 + b_conn;
    fprintf(f, "        <DataArray type=\"Int64\" Name=\"offsets\" format=\"appended\" offset=\"%llu\"/>\n", (unsigned long long)off);
    off += 8 + b_offs;
    fprintf(f, "        <DataArray type=\"UInt8\" Name=\"types\" format=\"appended\" offset=\"%llu\"/>\n", (unsigned long long)off);
    off += 8 + b_types;
    fprintf(f, "      </Cells>\n      <CellData>\n");
    for (int k = 0; k < nfields; k++) {
        char name[sizeof(fields[k].name) + 1];
        memcpy(name, fields[k].name, sizeof(fields[k].name));
        name[sizeof(fields[k].name)] = 0;
        for (char *q = name; *q; q++)
            if (*q == '"' || *q == '<' || *q == '>' || *q == '&') *q = '_';
        fprintf(f, "        <DataArray type=\"Float64\" Name=\"%s\" format=\"appended\" offset=\"%llu\"/>\n", name,
                (unsigned long long)off);
        off += 8 + b_field;
    }
    fprintf(f, "      </CellData>\n    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding=\"raw\">\n   _");
    int bad = write_block(f, pts, b_pts) || write_block(f, conn, b_conn) || write_block(f, offs, b_offs) ||
              write_block(f, types, b_types);
    for (int k = 0; k < nfields && !bad; k++) bad = write_block(f, values + (size_t)k * ncells, b_field);
    fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
    bad = bad || ferror(f);
    fclose(f);
    free(pts); free(conn); free(offs); free(types);
    return bad ? CIPHER_E_ARG : CIPHER_OK;
}
