// C wrapper around the reference's own STAR reader (MetaDataTable, src/metadata_table.cpp),
// compiled from the reference's sources into oracle/_ref/libstar_ref.so as the parity
// checker of the library's STAR parser.  Test infrastructure, never shipped.
#include "src/metadata_table.h"
#include <cstring>
#include <string>

// globals the reference defines in files outside the STAR reader (pipeline control,
// generated version string); nothing here reads them
std::string pipeline_control_outputname;
const char* g_RELION_VERSION = "reference";

static MetaDataTable* g_tab = nullptr;

extern "C" {

// Read data block `block` of `fn`; returns the number of rows or -1.
int ref_star_read(const char* fn, const char* block)
{
    try {
        delete g_tab;
        g_tab = new MetaDataTable();
        g_tab->read(fn, block);
        return (int)g_tab->numberOfObjects();
    } catch (...) {
        return -1;
    }
}

// Value of label `name` in row `i` as a double (int, bool and double labels); -2 if absent.
int ref_star_get_double(const char* name, long i, double* out)
{
    try {
        const EMDLabel l = EMDL::str2Label(name);
        if (l == EMDL_UNDEFINED || !g_tab || !g_tab->containsLabel(l)) return -2;
        if (EMDL::isInt(l)) {
            int v = 0;
            g_tab->getValue(l, v, i);
            *out = v;
        } else if (EMDL::isBool(l)) {
            bool v = false;
            g_tab->getValue(l, v, i);
            *out = v ? 1. : 0.;
        } else {
            double v = 0.;
            g_tab->getValue(l, v, i);
            *out = v;
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

// Value of label `name` in row `i` as text; -2 if absent.
int ref_star_get_string(const char* name, long i, char* out, int cap)
{
    try {
        const EMDLabel l = EMDL::str2Label(name);
        if (l == EMDL_UNDEFINED || !g_tab || !g_tab->containsLabel(l)) return -2;
        std::string v;
        g_tab->getValueToString(l, v, i);
        std::strncpy(out, v.c_str(), cap - 1);
        out[cap - 1] = 0;
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
