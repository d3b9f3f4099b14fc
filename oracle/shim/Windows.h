#pragma once
// Minimal stand-in for <Windows.h> so the reference's Utils.cpp compiles on Linux
// inside the oracle recipe. Only ensureDirectory() uses these names; nothing on
// the reconstruction path calls it.
typedef unsigned long DWORD;
#define INVALID_FILE_ATTRIBUTES ((DWORD)-1)
#define FILE_ATTRIBUTE_DIRECTORY 0x10
#define FALSE 0
#define ERROR_ALREADY_EXISTS 183
inline DWORD GetFileAttributesW(const wchar_t*) { return INVALID_FILE_ATTRIBUTES; }
inline int CreateDirectoryW(const wchar_t*, void*) { return 0; }
inline DWORD GetLastError() { return 0; }
