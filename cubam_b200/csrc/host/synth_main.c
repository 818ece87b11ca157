/* Command-line form of the synthetic BAM generator (synth.c): writes one file in a process of its own.
 *
 *   cubam_synth PATH SHAPE N_RECORDS SEED LEVEL STORED_FRAC N_BARCODES N_THREADS
 *
 * prints "record_bytes members file_bytes" and exits 0, or exits 1 when the file cannot be written.
 * A benchmark process that must not map the decoder's libraries (the timed CPU arm) makes its
 * input this way. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

int synth_bam(const char* path, int shape, int64_t n_records, uint64_t seed, int level, double stored_frac,
              int n_barcodes, int n_threads, int64_t* out_record_bytes, int64_t* out_members,
              int64_t* out_file_bytes);

int main(int argc, char** argv) {
    if (argc != 9) {
        fprintf(stderr, "usage: %s PATH SHAPE N_RECORDS SEED LEVEL STORED_FRAC N_BARCODES N_THREADS\n", argv[0]);
        return 2;
    }
    int64_t rb = 0, mb = 0, fb = 0;
    int rc = synth_bam(argv[1], atoi(argv[2]), strtoll(argv[3], NULL, 10), strtoull(argv[4], NULL, 10), atoi(argv[5]),
                       strtod(argv[6], NULL), atoi(argv[7]), atoi(argv[8]), &rb, &mb, &fb);
    if (rc) {
        fprintf(stderr, "cannot write %s\n", argv[1]);
        return 1;
    }
    printf("%lld %lld %lld\n", (long long)rb, (long long)mb, (long long)fb);
    return 0;
}
