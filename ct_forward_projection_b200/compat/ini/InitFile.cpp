// InitFile.cpp — implementation of the INI reader/writer (see InitFile.h).
#include "InitFile.h"

#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <utility>
#include <vector>

struct CInitFile::Store {
    struct Entry {
        std::string key, value, comment;
    };
    struct Section {
        std::string name;
        std::vector<Entry> entries;
    };
    std::vector<Section> sections;

    Section* find(const std::string& name)
    {
        for (auto& s : sections)
            if (s.name == name) return &s;
        return nullptr;
    }
    const Section* find(const std::string& name) const
    {
        for (auto& s : sections)
            if (s.name == name) return &s;
        return nullptr;
    }
};

namespace {

std::string trim(const std::string& s)
{
    const char* ws = " \t\r\n";
    const size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) return std::string();
    const size_t b = s.find_last_not_of(ws);
    return s.substr(a, b - a + 1);
}

template <typename T>
bool parse_number(const std::string& text, T& out)
{
    if (text.empty()) return false;
    const char* p = text.c_str();
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(p, &end);
    if (end == p || errno == ERANGE) return false;
    out = static_cast<T>(v);
    return true;
}

template <typename T>
BOOL get_number(const CInitFile* self, bool found, const std::string& text, T dflt, T& out)
{
    (void)self;
    if (found && parse_number(text, out)) return 1;
    out = dflt;
    return 0;
}

}  // namespace

CInitFile::CInitFile() : m_store(new Store) {}
CInitFile::~CInitFile() = default;

void CInitFile::GetFileName(LPSTR1 szFileName)
{
    m_store.reset(new Store);
    m_path = szFileName ? szFileName : "";
    std::ifstream in(m_path);
    if (!in) return;
    std::string line;
    Store::Section* cur = nullptr;
    while (std::getline(in, line)) {
        std::string t = trim(line);
        if (t.empty() || t[0] == ';' || t[0] == '#') continue;
        if (t[0] == '[') {
            const size_t close = t.find(']');
            const std::string name = trim(t.substr(1, close == std::string::npos ? std::string::npos : close - 1));
            cur = m_store->find(name);
            if (!cur) {
                m_store->sections.push_back(Store::Section{name, {}});
                cur = &m_store->sections.back();
            }
            continue;
        }
        const size_t eq = t.find('=');
        if (eq == std::string::npos || !cur) continue;
        Store::Entry e;
        e.key = trim(t.substr(0, eq));
        std::string rest = t.substr(eq + 1);
        const size_t semi = rest.find(';');
        if (semi != std::string::npos) {
            e.comment = rest.substr(semi);
            rest = rest.substr(0, semi);
        }
        e.value = trim(rest);
        bool replaced = false;
        for (auto& old : cur->entries)
            if (old.key == e.key) {
                old = e;
                replaced = true;
            }
        if (!replaced) cur->entries.push_back(e);
    }
}

void CInitFile::creatFile(LPSTR1 szFileName)
{
    m_store.reset(new Store);
    m_path = szFileName ? szFileName : "";
    std::ofstream out(m_path);
}

void CInitFile::SaveFile(LPSTR1 szFileName)
{
    const std::string path = szFileName ? std::string(szFileName) : m_path;
    std::ofstream out(path);
    for (const auto& s : m_store->sections) {
        out << "[" << s.name << "]\n";
        for (const auto& e : s.entries) out << e.key << "=" << e.value << (e.comment.empty() ? "" : "\t") << e.comment << "\n";
        out << "\n";
    }
}

bool CInitFile::lookup(LPSTR1 section, LPSTR1 key, std::string& out) const
{
    if (!section || !key) return false;
    const Store::Section* s = m_store->find(section);
    if (!s) return false;
    for (const auto& e : s->entries)
        if (e.key == key) {
            out = e.value;
            return true;
        }
    return false;
}

BOOL CInitFile::set(LPSTR1 section, LPSTR1 key, const std::string& value)
{
    if (!section || !key) return 0;
    Store::Section* s = m_store->find(section);
    if (!s) {
        m_store->sections.push_back(Store::Section{section, {}});
        s = &m_store->sections.back();
    }
    for (auto& e : s->entries)
        if (e.key == key) {
            e.value = value;
            return 1;
        }
    s->entries.push_back(Store::Entry{key, value, ""});
    return 1;
}

BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, LPSTR1 dflt, String& out)
{
    std::string v;
    if (lookup(sec, key, v)) {
        out = v;
        return 1;
    }
    out = dflt ? dflt : "";
    return 0;
}

BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, int dflt, char& out)
{
    std::string v;
    const bool f = lookup(sec, key, v);
    return get_number<char>(this, f, v, (char)dflt, out);
}
BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, int dflt, short& out)
{
    std::string v;
    const bool f = lookup(sec, key, v);
    return get_number<short>(this, f, v, (short)dflt, out);
}
BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, int dflt, int& out)
{
    std::string v;
    const bool f = lookup(sec, key, v);
    return get_number<int>(this, f, v, dflt, out);
}
BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, long dflt, long& out)
{
    std::string v;
    const bool f = lookup(sec, key, v);
    return get_number<long>(this, f, v, dflt, out);
}
BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, double dflt, double& out)
{
    std::string v;
    const bool f = lookup(sec, key, v);
    return get_number<double>(this, f, v, dflt, out);
}
BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, __int64 dflt, __int64& out)
{
    std::string v;
    const bool f = lookup(sec, key, v);
    return get_number<__int64>(this, f, v, dflt, out);
}
BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, size_t dflt, size_t& out)
{
    std::string v;
    const bool f = lookup(sec, key, v);
    return get_number<size_t>(this, f, v, dflt, out);
}
BOOL CInitFile::GetEntryValue(LPSTR1 sec, LPSTR1 key, float dflt, float& out)
{
    std::string v;
    const bool f = lookup(sec, key, v);
    return get_number<float>(this, f, v, dflt, out);
}

namespace {
template <typename T>
std::string num_text(T v)
{
    std::ostringstream os;
    os.precision(9);
    os << v;
    return os.str();
}
}  // namespace

BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, String v) { return set(s, k, v); }
BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, char v) { return set(s, k, num_text((int)v)); }
BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, short v) { return set(s, k, num_text(v)); }
BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, int v) { return set(s, k, num_text(v)); }
#ifdef _WIN32
BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, unsigned long v) { return set(s, k, num_text(v)); }
#endif
BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, double v) { return set(s, k, num_text(v)); }
BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, __int64 v) { return set(s, k, num_text(v)); }
BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, size_t v) { return set(s, k, num_text(v)); }
BOOL CInitFile::SetEntryValue(LPSTR1 s, LPSTR1 k, float v) { return set(s, k, num_text(v)); }
