// InitFile.h — key=value INI reader/writer with the interface of the
// reference's CInitFile (Shared/Include/InitFile.h:40-104), written from that
// header's declarations and the syntax of Config/ScanSetting.ini and
// Config/OutPutFolder.ini:
//   [Section]
//   Key=Value        ; comment       (the value ends at the first ';', trimmed)
//   ; comment line
// Lookups of a missing file, section or key return FALSE and store the given
// default, which is how the reference detects missing entries
// (ForwardProjection.cpp:209-225 compares against -100 / "null").
#pragma once

#include <cstddef>
#include <memory>
#include <string>

#ifndef BOOL
typedef int BOOL;
#endif
typedef const char* LPSTR1;
typedef std::string String;
#ifndef _WIN32
typedef long long __int64;
#endif

class CInitFile {
public:
    CInitFile();
    ~CInitFile();
    CInitFile(const CInitFile&) = delete;
    CInitFile& operator=(const CInitFile&) = delete;

    // Loads and parses szFileName (InitFile.h:65).
    void GetFileName(LPSTR1 szFileName = "Reconstruct.txt");
    // Writes the entries back, to szFileName or to the loaded file (InitFile.h:66).
    void SaveFile(LPSTR1 szFileName = 0);
    String GetParaFilePath() { return m_path; }
    void creatFile(LPSTR1 szFileName);

    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, String szValue);
    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, char iValue);
    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, short iValue);
    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, int iValue);
#ifdef _WIN32
    // distinct from size_t only where unsigned long is 32-bit
    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, unsigned long iValue);
#endif
    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, double dbValue);
    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, __int64 i64value);
    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, size_t iValue);
    BOOL SetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, float iValue);

    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, LPSTR1 szDefault, String& szValue);
    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, int iDefault, char& iValue);
    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, int iDefault, short& iValue);
    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, int iDefault, int& iValue);
    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, long iDefault, long& iValue);
    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, double dbDefault, double& dbValue);
    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, __int64 i64Default, __int64& i64Value);
    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, size_t iDefault, size_t& iValue);
    BOOL GetEntryValue(LPSTR1 szSection, LPSTR1 szEntry, float iDefault, float& iValue);

private:
    struct Store;
    bool lookup(LPSTR1 section, LPSTR1 key, std::string& out) const;
    BOOL set(LPSTR1 section, LPSTR1 key, const std::string& value);
    std::unique_ptr<Store> m_store;
    std::string m_path;
};
