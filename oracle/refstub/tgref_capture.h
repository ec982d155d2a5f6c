// TEST INFRASTRUCTURE ONLY: access to what the single-rank stand-ins captured.
#ifndef TGREF_CAPTURE_H
#define TGREF_CAPTURE_H

void tgref_set_quiet(bool quiet);            // PetscPrintf / PetscFPrintf output on or off
void tgref_matrix_clear();                   // forget the captured HYPRE_IJMatrixSetValues rows
long tgref_matrix_rows();                    // rows captured (largest row id + 1)
long tgref_matrix_nnz();                     // entries captured
void tgref_matrix_csr(long *rowptr, long *col, double *val);
// the number printed after `prefix` in the last PetscPrintf message that starts
// with it (messages are recorded whether or not they are shown)
bool tgref_printed_value(const char *prefix, double *value);

#endif
