/* Drop-in comm_buffer (reference buffer.hh:16-44).  The device library owns
 * all working memory, so this is a host scratch holder kept for the
 * constructor signatures multigrid(p, gm, com) and region(p, gm, com). */
#ifndef PGMG_BUFFER_HH
#define PGMG_BUFFER_HH

#include <cstdlib>

class comm_buffer {
   public:
    double* buf;
    size_t mem;
    comm_buffer() : buf(0), mem(0) {}
    ~comm_buffer() { std::free(buf); }
    inline void check_buf(int q) { reallocate(q * sizeof(double)); }
    inline void check_buf_int(int q) { reallocate(q * sizeof(int)); }
    inline void check_buf_float(int q) { reallocate(q * sizeof(float)); }

   private:
    void reallocate(size_t n) {
        if (n > mem) {
            std::free(buf);
            buf = static_cast<double*>(std::malloc(n));
            mem = n;
        }
    }
    comm_buffer(const comm_buffer&);
    comm_buffer& operator=(const comm_buffer&);
};

#endif
