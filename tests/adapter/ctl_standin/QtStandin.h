// Stand-in for the few Qt Core names that the CTL adapter and CTL's headers
// use (QVariant, QVariantMap, QSize, QSizeF, qCritical/qWarning, emit), so the
// adapter compiles and runs in this test without Qt.  Test code only.
#ifndef CTL_STANDIN_QT_H
#define CTL_STANDIN_QT_H

#include <cstdio>
#include <map>
#include <memory>
#include <sstream>
#include <string>

#define emit

class QVariant;
class QVariantMap
{
public:
    void insert(const std::string& key, const QVariant& value);
    QVariant value(const std::string& key, const QVariant& fallback) const;
    QVariant value(const std::string& key) const;
    bool contains(const std::string& key) const { return _m.count(key) != 0; }

private:
    std::map<std::string, std::shared_ptr<QVariant>> _m;
};

class QVariant
{
public:
    QVariant() = default;
    QVariant(bool v) : _kind(1), _d(v ? 1.0 : 0.0) {}
    QVariant(int v) : _kind(2), _d(v) {}
    QVariant(unsigned v) : _kind(2), _d(v) {}
    QVariant(float v) : _kind(3), _d(v) {}
    QVariant(double v) : _kind(3), _d(v) {}
    QVariant(const char* s) : _kind(4), _s(s) {}
    QVariant(const QVariantMap& m) : _kind(5), _map(std::make_shared<QVariantMap>(m)) {}
    bool isValid() const { return _kind != 0; }
    bool toBool() const { return _d != 0.0; }
    int toInt() const { return int(_d); }
    unsigned toUInt() const { return unsigned(_d); }
    float toFloat() const { return float(_d); }
    double toDouble() const { return _d; }
    std::string toString() const { return _s; }
    QVariantMap toMap() const { return _map ? *_map : QVariantMap(); }

private:
    int _kind = 0;
    double _d = 0.0;
    std::string _s;
    std::shared_ptr<QVariantMap> _map;
};

inline void QVariantMap::insert(const std::string& key, const QVariant& value)
{
    _m[key] = std::make_shared<QVariant>(value);
}
inline QVariant QVariantMap::value(const std::string& key, const QVariant& fallback) const
{
    auto it = _m.find(key);
    return it == _m.end() ? fallback : *it->second;
}
inline QVariant QVariantMap::value(const std::string& key) const { return value(key, QVariant()); }

class QSize
{
public:
    QSize(int w = 0, int h = 0) : _w(w), _h(h) {}
    int width() const { return _w; }
    int height() const { return _h; }

private:
    int _w, _h;
};

class QSizeF
{
public:
    QSizeF(double w = 0.0, double h = 0.0) : _w(w), _h(h) {}
    double width() const { return _w; }
    double height() const { return _h; }

private:
    double _w, _h;
};

// qCritical() << ... / qWarning() << ...: one line on stderr per statement
class QDebugStandin
{
public:
    explicit QDebugStandin(const char* level) { _s << level << ": "; }
    ~QDebugStandin() { std::fprintf(stderr, "%s\n", _s.str().c_str()); }
    template <typename T>
    QDebugStandin& operator<<(const T& v)
    {
        _s << v << ' ';
        return *this;
    }

private:
    std::ostringstream _s;
};
inline QDebugStandin qCritical() { return QDebugStandin("critical"); }
inline QDebugStandin qWarning() { return QDebugStandin("warning"); }
inline QDebugStandin qDebug() { return QDebugStandin("debug"); }

#endif
