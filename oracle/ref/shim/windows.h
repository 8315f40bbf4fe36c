/* Header shim for compiling the reference's CPU query path on Linux.
 * The reference includes <Windows.h> under WIN32 only for these typedefs;
 * nothing from the Win32 API is called on the query path. */
#ifndef ENC_ORACLE_SHIM_WINDOWS_H
#define ENC_ORACLE_SHIM_WINDOWS_H
typedef unsigned int DWORD;
typedef int BOOL;
#endif
