/* Error reporting of the reference CPU objects that the reference extension
 * links beside the drop-in library (oracle/Makefile, target `refext`).
 *
 * Test infrastructure only.  The reference's CPU solvers report failures
 * through _disptools_set_error (src/headers/disptools.h:204-240); its own
 * definition (src/disptools.c:10-24) writes a state of its own, which the
 * extension would never read, because the extension's disptools_has_error()
 * and disptools_get_error() are the drop-in's.  This definition writes the
 * drop-in's state instead, so the extension sees failures of either side. */
#include <stdbool.h>
#include <string.h>

#include "disptools.h"

static void copy_field(char *dst, const char *src, size_t n) {
    strncpy(dst, src ? src : "", n - 1);
    dst[n - 1] = '\0';
}

void _disptools_set_error(const bool error, const int line, const char file[512], const char function[512],
                          const char message[1024], const char trace[4096]) {
    disptools_error_state *e = disptools_get_error();
    e->error = error;
    e->line = line;
    copy_field(e->file, file, sizeof e->file);
    copy_field(e->function, function, sizeof e->function);
    copy_field(e->message, message, sizeof e->message);
    copy_field(e->trace, trace, sizeof e->trace);
}
