/* PGMG-compatible communication buffer for the CPU oracle build (test
 * infrastructure): a growable scratch array of doubles. */
#ifndef RMT3D_ORACLE_PGMG_BUFFER_HH
#define RMT3D_ORACLE_PGMG_BUFFER_HH
#include <cstddef>

struct comm_buffer {
    double *buf;
    size_t mem;
    comm_buffer() : buf(nullptr), mem(0) {}
    ~comm_buffer() { delete[] buf; }
    comm_buffer(const comm_buffer &) = delete;
    comm_buffer &operator=(const comm_buffer &) = delete;
    void check_buf(size_t n) {
        if (n <= mem) return;
        delete[] buf;
        mem = n;
        buf = new double[mem];
    }
    void check_buf_uint(size_t n) { check_buf((n * sizeof(unsigned int) + sizeof(double) - 1) / sizeof(double)); }
};
#endif
