/*
 * oracle/ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Builds the UNMODIFIED reference PAR_Word2Vec_cpu.cpp (path given by -DREF_SOURCE,
 * read where it lies; nothing is copied into this repository) into a binary that
 * also dumps the reference's globals after training, so that tests can compare
 * bit patterns instead of the 6-decimal text output:
 *
 *   par_w2v_ref <reference flags ...> -dump <prefix> [-dump-table 1]
 *
 * writes   <prefix>.meta      "vocab_size hidden_size train_words file_size"
 *          <prefix>.vocab     one "word count" line per vocab entry (vocab order)
 *          <prefix>.win       final W_in,  vocab_size*hidden_size float32
 *          <prefix>.wout      final W_out, vocab_size*hidden_size float32
 *          <prefix>.exptable  expTable[1001] float32   (PAR_Word2Vec_cpu.cpp:822-826)
 *          <prefix>.win0      W_in as InitNet leaves it (PAR_Word2Vec_cpu.cpp:337-357)
 *          <prefix>.table     the 1e8-entry unigram table int32 (only with -dump-table 1,
 *                             PAR_Word2Vec_cpu.cpp:96-117)
 *          <prefix>.load      seconds of the training region's corpus load alone (only with
 *                             -time-load 1): the same per-thread fopen/fseek/loadStream the
 *                             reference runs at the start of its timed region
 *                             (PAR_Word2Vec_cpu.cpp:398-416), timed with its rtclock()
 *
 * The reference's main() runs first exactly as the reference binary would
 * (PAR_Word2Vec_cpu.cpp:739-842), including its "PAR_Word2Vec_cpu_time" file
 * (written into the current directory) and its -output file.
 */
#define main parw2v_reference_main
#include REF_SOURCE
#undef main

#include <cstdio>
#include <cstdlib>
#include <cstring>

static int dump_raw(const char *prefix, const char *ext, const void *p, size_t bytes) {
    char path[4096];
    snprintf(path, sizeof(path), "%s%s", prefix, ext);
    FILE *f = fopen(path, "wb");
    if (!f) {
        fprintf(stderr, "ref_driver: cannot open %s\n", path);
        return 1;
    }
    size_t w = fwrite(p, 1, bytes, f);
    fclose(f);
    return w == bytes ? 0 : 1;
}

int main(int argc, char **argv) {
    const char *prefix = NULL;
    int dump_table = 0, time_load = 0;
    for (int a = 1; a + 1 < argc; a++) {
        if (!strcmp(argv[a], "-dump")) prefix = argv[a + 1];
        if (!strcmp(argv[a], "-dump-table")) dump_table = atoi(argv[a + 1]);
        if (!strcmp(argv[a], "-time-load")) time_load = atoi(argv[a + 1]);
    }
    int rc = parw2v_reference_main(argc, argv);
    if (rc != 0 || prefix == NULL || argc == 1 || output_file[0] == 0) return rc;

    const size_t n = (size_t) vocab_size * (size_t) hidden_size;
    char path[4096];
    snprintf(path, sizeof(path), "%s.meta", prefix);
    FILE *f = fopen(path, "w");
    if (!f) return 1;
    fprintf(f, "%d %d %llu %llu\n", vocab_size, hidden_size, (unsigned long long) train_words,
            (unsigned long long) file_size);
    fclose(f);
    snprintf(path, sizeof(path), "%s.vocab", prefix);
    f = fopen(path, "wb");
    if (!f) return 1;
    for (int i = 0; i < vocab_size; i++) fprintf(f, "%s %u\n", vocab[i].word, vocab[i].cn);
    fclose(f);
    int bad = 0;
    bad |= dump_raw(prefix, ".win", W_in, n * sizeof(float));
    bad |= dump_raw(prefix, ".wout", W_out, n * sizeof(float));
    bad |= dump_raw(prefix, ".exptable", expTable, (EXP_TABLE_SIZE + 1) * sizeof(float));
    if (dump_table) bad |= dump_raw(prefix, ".table", table, (size_t) table_size * sizeof(int));
    if (time_load && !disk) {
        /* the load phase of the reference's timed region on its own, with the reference's
           functions and the same per-thread split of the file */
        const double t0 = rtclock();
#pragma omp parallel num_threads(num_threads)
        {
            const int id = omp_get_thread_num();
            FILE *fin = fopen(train_file, "rb");
            if (fin) {
                fseek(fin, file_size * id / num_threads, SEEK_SET);
                ulonglong local = train_words / num_threads + (train_words % num_threads > 0 ? 1 : 0);
                int *stream = (int *) _mm_malloc((local + 1) * sizeof(int), 64);
                loadStream(fin, stream, local);
                fclose(fin);
                _mm_free(stream);
            }
        }
        const double secs = rtclock() - t0;
        snprintf(path, sizeof(path), "%s.load", prefix);
        f = fopen(path, "w");
        if (!f) return 1;
        fprintf(f, "%.6f\n", secs);
        fclose(f);
    }
    /* InitNet only depends on vocab_size and hidden_size: run it again for the initial W_in */
    InitNet();
    bad |= dump_raw(prefix, ".win0", W_in, n * sizeof(float));
    return bad;
}
