/* b200ode_io -- fast reader/writer for the reference's cell CSV files
 * (libb200ode_host.so; CPU only, no GPU needed).
 *
 * Format, as the reference's csvReader / csvWriter use it
 * (src/InputOutput/Reader/csvReader.cpp:28-159, Writer/csvWriter.cpp:29-110):
 * a header line naming the columns -- every column whose name contains "CO" is
 * a species mass fraction, "ENTHA" the specific enthalpy (optional), "TEMPE"
 * the temperature (required), "Points" the three coordinates (optional) -- then
 * one line per cell with the values in the order species..., [ENTHA], TEMPE,
 * [x, y, z].
 *
 * Differences from the reference, which parses line by line into one
 * vector<double> per cell (array of structures): the file is read in one piece
 * and parsed by `threads` threads straight into structure-of-arrays buffers with
 * the cell index innermost (the layout b200ode_integrate takes), and numbers are
 * written in their shortest exactly-round-tripping form (the reference writes 7
 * significant digits).  Files this writes are read by the reference's reader. */
#ifndef B200ODE_IO_H
#define B200ODE_IO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t n_cells;
    int32_t n_species;
    int32_t has_enthalpy;
    int32_t has_coordinates;
} b200ode_csv_info;

/* Header and line count of a cell CSV file.  0 on success, -1 on error
 * (message in b200ode_io_last_error). */
int b200ode_csv_inspect(const char* path, b200ode_csv_info* info);

/* Parse the file into caller buffers sized from b200ode_csv_inspect:
 * T[n], Y[nsp * n] (Y[k * n + c]), H[n] (or NULL), XYZ[3 * n] (XYZ[d * n + c],
 * or NULL).  threads <= 0 = all hardware threads.  0 on success, -1 on error
 * (malformed number, wrong column count, ...; the message names the line). */
int b200ode_csv_read(const char* path, int32_t threads, double* T, double* Y, double* H, double* XYZ);

/* Write n cells in the reference's column order; H and XYZ may be NULL (no
 * such columns).  0 on success, -1 on error. */
int b200ode_csv_write(const char* path, int64_t n_cells, int32_t n_species, const double* T, const double* Y,
                      const double* H, const double* XYZ, int32_t threads);

/* Message of the last I/O error on this thread ("" if none). */
const char* b200ode_io_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* B200ODE_IO_H */
