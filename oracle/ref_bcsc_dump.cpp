// Checker harness (TEST INFRASTRUCTURE): runs the reference's own COO reader and
// BCSC builder, compiled from the reference's sources where they lie
// (src/utils/matrix.h: COOMatrix(file, 1, true) :270-303 and
// BCSRCSCMatrix(coo, 16, 16) :1356 -> coo2bcsc :1200-1269), and writes the
// resulting bcsc arrays so the oracle's restatement can be compared with them.
//
// usage: ref_bcsc_dump <coo.tsv> <blocksize> <out.bin>
// out.bin: int32 n_col_ptr, col_ptr[n]; int32 n_blocks, row_index[n];
//          int32 n_col_index, col_index[n]; float values[n_blocks*bs*bs]
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "utils/matrix.h"

static void put_ints(FILE *f, const std::vector<int> &v) {
    int n = (int)v.size();
    fwrite(&n, sizeof(int), 1, f);
    if (n) fwrite(v.data(), sizeof(int), (size_t)n, f);
}

int main(int argc, char **argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s coo.tsv blocksize out.bin\n", argv[0]);
        return 2;
    }
    std::string file(argv[1]);
    int bs = atoi(argv[2]);
    ftxj::COOMatrix coo(file, 1, true);
    ftxj::BCSRCSCMatrix m(coo, bs, bs);
    FILE *f = fopen(argv[3], "wb");
    if (!f) return 1;
    put_ints(f, m.bcsc_len_);
    put_ints(f, m.bcsc_row_index_);
    put_ints(f, m.bcsc_col_index_);
    fwrite(m.bcsc_values_.data(), sizeof(float), m.bcsc_values_.size(), f);
    fclose(f);
    return 0;
}
