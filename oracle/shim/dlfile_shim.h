/*
 * dlfile_shim.h -- the file helpers of the un-vendored `domlib` that the
 * reference's src/io.c calls (dl_open_file, dl_get_next_line, ...), written
 * for this project from those call sites.  TEST INFRASTRUCTURE ONLY: it lets
 * src/io.c compile unmodified into oracle/_ref so the CSR / grid readers and
 * writers can be checked against the reference's own parsing code.
 *
 * Assumed semantics (the call sites rely on no more than this):
 *  - dl_get_next_line reads one line, drops its trailing newline, returns its
 *    length (0 for a blank line) or -1 at end of file; a last line without a
 *    newline still counts, and the newline that ends the file opens no extra
 *    line;
 *  - dl_get_ne_str counts whitespace-separated tokens;
 *  - dl_reset_file rewinds, dl_mark_file / dl_restore_file save and return to a
 *    position.
 */
#ifndef GB_ORACLE_DLFILE_SHIM_H
#define GB_ORACLE_DLFILE_SHIM_H

#include <errno.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>

typedef struct {
  FILE * fd;
  long mark;
} file_t;

enum {
  DL_FILE_SUCCESS = 1,
  DL_FILE_BAD_PARAMETERS,
  DL_FILE_PATH_PARSE_FAILURE,
  DL_FILE_PATH_BAD,
  DL_FILE_PATH_ACCESS_DENIED,
  DL_FILE_READ_ACCESS_DENIED,
  DL_FILE_WRITE_ACCESS_DENIED,
  DL_FILE_OPEN_FAILED
};

static inline int dl_open_file(const char * name, const char * mode, file_t ** out)
{
  FILE * fd;
  if (!name || !mode || !out) return DL_FILE_BAD_PARAMETERS;
  fd = fopen(name, mode);
  if (!fd) {
    if (errno == ENOENT || errno == ENOTDIR) return DL_FILE_PATH_BAD;
    if (errno == EACCES) return mode[0] == 'r' ? DL_FILE_READ_ACCESS_DENIED
                                               : DL_FILE_WRITE_ACCESS_DENIED;
    return DL_FILE_OPEN_FAILED;
  }
  *out = (file_t *)malloc(sizeof(file_t));
  (*out)->fd = fd;
  (*out)->mark = 0;
  return DL_FILE_SUCCESS;
}

static inline void dl_close_file(file_t * f)
{
  if (f) {
    fclose(f->fd);
    free(f);
  }
}

static inline void dl_reset_file(file_t * f) { rewind(f->fd); }
static inline void dl_mark_file(file_t * f) { f->mark = ftell(f->fd); }
static inline void dl_restore_file(file_t * f) { fseek(f->fd, f->mark, SEEK_SET); }

static inline ssize_t dl_get_next_line(file_t * f, char ** line, size_t * cap)
{
  ssize_t n = getline(line, cap, f->fd);
  if (n < 0) return -1;
  if (n > 0 && (*line)[n - 1] == '\n') (*line)[--n] = '\0';
  return n;
}

static inline size_t dl_get_ne_str(const char * s)
{
  size_t n = 0;
  int in = 0;
  for (; *s; ++s) {
    const int sp = (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\n' || *s == '\v' ||
                    *s == '\f');
    if (!sp && !in) ++n;
    in = !sp;
  }
  return n;
}

static inline int dl_fprintf(file_t * f, const char * fmt, ...)
{
  int r;
  va_list ap;
  va_start(ap, fmt);
  r = vfprintf(f->fd, fmt, ap);
  va_end(ap);
  return r;
}

static inline char * char_alloc(size_t n) { return (char *)malloc(n ? n : 1); }

#endif
