/* In-memory stand-in for the MATLAB runtime behind tests/mex_fake/mex.h, and
 * a driver that runs the gateway's mexFunction on commands read from a text
 * script: each line "command arg ..." where an argument is a scalar number, a
 * string in quotes, "@name" (a raw (rows, cols) double file name.bin with its
 * shape in name.shape), "#k" (the k-th output kept from an earlier line) or
 * "sparse:name" (name_ir/name_jc/name_pr files of a Q x N sparse matrix).
 * Every output k of a line is written to out_<line>_<k>.bin (doubles; cells
 * as one row per element; sparse as dense triplets).  A MATLAB error prints
 * "ERROR <id> <message>" and continues with the next line.  Test
 * infrastructure only. */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

struct mxArray_tag {
  mxClassID cls;
  size_t m, n;
  int sparse;
  void* data;           /* doubles, uint64s or chars */
  mwIndex *ir, *jc;     /* sparse */
  mxArray** cells;
};

static jmp_buf g_err;
static void (*g_exit)(void) = NULL;

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  char msg[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  printf("ERROR %s %s\n", id, msg);
  fflush(stdout);
  longjmp(g_err, 1);
}
int mexAtExit(void (*fn)(void)) { g_exit = fn; return 0; }
static mxArray* mk(mxClassID c, size_t m, size_t n, size_t esz) {
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = c; a->m = m; a->n = n;
  a->data = calloc((m * n) > 0 ? m * n : 1, esz);
  return a;
}
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) { (void)c; return mk(mxDOUBLE_CLASS, m, n, 8); }
mxArray* mxCreateDoubleScalar(double v) { mxArray* a = mk(mxDOUBLE_CLASS, 1, 1, 8); *(double*)a->data = v; return a; }
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity c) { (void)c; return mk(cls, m, n, 8); }
mxArray* mxCreateSparse(mwSize m, mwSize n, mwSize nz, mxComplexity c) {
  (void)c;
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = mxDOUBLE_CLASS; a->m = m; a->n = n; a->sparse = 1;
  a->data = calloc(nz ? nz : 1, 8);
  a->ir = (mwIndex*)calloc(nz ? nz : 1, sizeof(mwIndex));
  a->jc = (mwIndex*)calloc(n + 1, sizeof(mwIndex));
  return a;
}
mxArray* mxCreateCellMatrix(mwSize m, mwSize n) {
  mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
  a->cls = mxCELL_CLASS; a->m = m; a->n = n;
  a->cells = (mxArray**)calloc((m * n) > 0 ? m * n : 1, sizeof(mxArray*));
  return a;
}
void mxSetCell(mxArray* a, mwIndex i, mxArray* v) { a->cells[i] = v; }
void* mxGetData(const mxArray* a) { return a->data; }
double* mxGetPr(const mxArray* a) { return (double*)a->data; }
mwIndex* mxGetIr(const mxArray* a) { return a->ir; }
mwIndex* mxGetJc(const mxArray* a) { return a->jc; }
size_t mxGetM(const mxArray* a) { return a->m; }
size_t mxGetN(const mxArray* a) { return a->n; }
size_t mxGetNumberOfElements(const mxArray* a) { return a->m * a->n; }
double mxGetScalar(const mxArray* a) {
  return a->cls == mxUINT64_CLASS ? (double)*(uint64_t*)a->data : *(double*)a->data;
}
int mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
int mxIsUint64(const mxArray* a) { return a->cls == mxUINT64_CLASS; }
int mxIsComplex(const mxArray* a) { (void)a; return 0; }
int mxIsSparse(const mxArray* a) { return a->sparse; }
int mxIsChar(const mxArray* a) { return a->cls == mxCHAR_CLASS; }
int mxGetString(const mxArray* a, char* buf, mwSize len) {
  if (a->cls != mxCHAR_CLASS || strlen((char*)a->data) + 1 > len) return 1;
  strcpy(buf, (char*)a->data);
  return 0;
}
void* mxMalloc(size_t n) { return malloc(n ? n : 1); }
void* mxCalloc(size_t n, size_t s) { return calloc(n ? n : 1, s ? s : 1); }
void mxFree(void* p) { free(p); }

static mxArray* load_dense(const char* name) {
  char path[512];
  size_t m = 0, n = 0;
  snprintf(path, sizeof path, "%s.shape", name);
  FILE* f = fopen(path, "r");
  if (!f || fscanf(f, "%zu %zu", &m, &n) != 2) { fprintf(stderr, "bad shape %s\n", name); exit(2); }
  fclose(f);
  mxArray* a = mxCreateDoubleMatrix(m, n, mxREAL);
  snprintf(path, sizeof path, "%s.bin", name);
  f = fopen(path, "rb");
  if (!f || fread(a->data, 8, m * n, f) != m * n) { fprintf(stderr, "bad data %s\n", name); exit(2); }
  fclose(f);
  return a;
}
static mxArray* load_sparse(const char* name) {
  char nm[512];
  snprintf(nm, sizeof nm, "%s_pr", name);
  mxArray* pr = load_dense(nm);
  snprintf(nm, sizeof nm, "%s_ir", name);
  mxArray* ir = load_dense(nm);
  snprintf(nm, sizeof nm, "%s_jc", name);
  mxArray* jc = load_dense(nm);
  snprintf(nm, sizeof nm, "%s_mn", name);
  mxArray* mn = load_dense(nm);
  const size_t nz = pr->m * pr->n, ncol = (size_t)((double*)mn->data)[1];
  mxArray* s = mxCreateSparse((size_t)((double*)mn->data)[0], ncol, nz, mxREAL);
  for (size_t k = 0; k < nz; ++k) {
    ((double*)s->data)[k] = ((double*)pr->data)[k];
    s->ir[k] = (mwIndex)((double*)ir->data)[k];
  }
  for (size_t j = 0; j <= ncol; ++j) s->jc[j] = (mwIndex)((double*)jc->data)[j];
  return s;
}
static void dump(const mxArray* a, int line, int k) {
  char path[64];
  snprintf(path, sizeof path, "out_%d_%d.bin", line, k);
  FILE* f = fopen(path, "wb");
  if (a->cls == mxCELL_CLASS) {
    for (size_t i = 0; i < a->m * a->n; ++i) {
      const mxArray* c = a->cells[i];
      const double cnt = (double)(c->m * c->n);
      fwrite(&cnt, 8, 1, f);
      fwrite(c->data, 8, c->m * c->n, f);
    }
  } else if (a->sparse) {
    for (size_t j = 0; j < a->n; ++j)
      for (mwIndex p = a->jc[j]; p < a->jc[j + 1]; ++p) {
        const double t[3] = {(double)a->ir[p], (double)j, ((double*)a->data)[p]};
        fwrite(t, 8, 3, f);
      }
  } else if (a->cls == mxUINT64_CLASS) {
    const double v = 1.0;  /* a handle: only its presence is recorded */
    fwrite(&v, 8, 1, f);
  } else {
    fwrite(a->data, 8, a->m * a->n, f);
  }
  fclose(f);
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  FILE* s = fopen(argv[1], "r");
  if (!s) return 2;
  char lineb[4096];
  mxArray* kept[64] = {0};
  int nkept = 0, line = 0;
  while (fgets(lineb, sizeof lineb, s)) {
    const mxArray* in[16];
    mxArray* out[8] = {0};
    int nin = 0, nout = 1;
    char* tok = strtok(lineb, " \t\n");
    if (!tok) continue;
    nout = atoi(tok);
    while ((tok = strtok(NULL, " \t\n")) && nin < 16) {
      if (tok[0] == '"') {
        mxArray* a = mk(mxCHAR_CLASS, 1, strlen(tok), 1);
        memcpy(a->data, tok + 1, strlen(tok) - 2);
        in[nin++] = a;
      } else if (tok[0] == '@') {
        in[nin++] = load_dense(tok + 1);
      } else if (!strncmp(tok, "sparse:", 7)) {
        in[nin++] = load_sparse(tok + 7);
      } else if (tok[0] == '#') {
        in[nin++] = kept[atoi(tok + 1)];
      } else {
        in[nin++] = mxCreateDoubleScalar(atof(tok));
      }
    }
    if (!setjmp(g_err)) {
      mexFunction(nout, out, nin, in);
      for (int k = 0; k < nout; ++k)
        if (out[k]) dump(out[k], line, k);
      if (nkept < 64) kept[nkept++] = out[0] ? out[0] : mxCreateDoubleScalar(0.0);
      printf("OK %d\n", line);
    } else if (nkept < 64) {
      kept[nkept++] = mxCreateDoubleScalar(0.0);  /* keeps output numbering aligned with lines */
    }
    fflush(stdout);
    ++line;
  }
  fclose(s);
  if (g_exit) g_exit();
  return 0;
}
