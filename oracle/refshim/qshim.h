// qshim.h -- the few Qt types and macros the reference's kMC sources use,
// restated over the C++ standard library so that those sources compile here
// unchanged (TEST INFRASTRUCTURE: oracle/refshim builds the reference's own
// World, Grid, Potential, Random and agent classes into oracle/_ref/ as the
// checker of the kMC step; nothing in the product links it).
//
// Only what the compiled files need is here, with Qt's meaning where it
// matters to them: QList/QVector are int-indexed sequences, QString a text
// value with arg() substitution, qFatal throws (the harness reports it),
// qDebug discards its output, foreach iterates a container.
#pragma once

#include <algorithm>
#include <cmath>
// Qt's own headers include <math.h>, which (libstdc++) puts the floating-point
// overloads of abs in the global namespace; the reference's unqualified
// abs(double) calls (potential.cpp:212) rely on that.
#include <math.h>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

typedef uint64_t quint64;
typedef int64_t qint64;
typedef uint32_t quint32;
typedef int32_t qint32;
typedef uint8_t quint8;
typedef double qreal;

class QMetaEnum {
public:
    const char* valueToKey(int) const { return "?"; }
};
class QMetaObject {
public:
    int indexOfEnumerator(const char*) const { return 0; }
    QMetaEnum enumerator(int) const { return QMetaEnum(); }
};

#define Q_OBJECT \
public:          \
    static const QMetaObject staticMetaObject; \
private:
#define Q_DISABLE_COPY(C) \
    C(const C&) = delete; \
    C& operator=(const C&) = delete;
#define Q_ENUMS(x)
#define Q_CHECK_PTR(p) ((void)(p))
#define signals public
#define slots
#define emit
#define foreach(decl, container) for (decl : container)

class QString {
public:
    QString() {}
    QString(const char* s) : m_s(s ? s : "") {}
    QString(const std::string& s) : m_s(s) {}
    const std::string& toStdString() const { return m_s; }
    bool operator==(const QString& o) const { return m_s == o.m_s; }
    bool operator!=(const QString& o) const { return m_s != o.m_s; }
    bool operator==(const char* o) const { return m_s == o; }
    bool operator!=(const char* o) const { return m_s != o; }
    QString operator+(const QString& o) const { return QString(m_s + o.m_s); }
    QString& operator+=(const QString& o) { m_s += o.m_s; return *this; }
    int size() const { return (int)m_s.size(); }
    int length() const { return (int)m_s.size(); }
    bool isEmpty() const { return m_s.empty(); }
    QString at(int i) const { return QString(m_s.substr((size_t)i, 1)); }
    QString toLower() const {
        std::string t = m_s;
        for (char& c : t) c = (char)std::tolower((unsigned char)c);
        return QString(t);
    }
    // arg(): replaces the lowest-numbered %n marker by the value
    template <class T>
    QString arg(const T& v, int = 0, int = 0, int = 0) const {
        std::ostringstream o;
        o << v;
        return subst(o.str());
    }
    QString arg(const QString& v, int = 0) const { return subst(v.m_s); }
    QString arg(double v, int = 0, char = 'g', int = -1) const {
        std::ostringstream o;
        o << v;
        return subst(o.str());
    }
    static QString number(double v) {
        std::ostringstream o;
        o << v;
        return QString(o.str());
    }

private:
    QString subst(const std::string& v) const {
        for (char d = '1'; d <= '9'; ++d) {
            const std::string key = std::string("%") + d;
            const size_t p = m_s.find(key);
            if (p != std::string::npos) {
                std::string t = m_s;
                t.replace(p, 2, v);
                return QString(t);
            }
        }
        return *this;
    }
    std::string m_s;
};
inline std::ostream& operator<<(std::ostream& o, const QString& s) { return o << s.toStdString(); }
#define qPrintable(s) ((s).toStdString().c_str())

template <class T>
class QVector {
public:
    QVector() {}
    explicit QVector(int n) : m_v((size_t)std::max(n, 0)) {}
    QVector(int n, const T& v) : m_v((size_t)std::max(n, 0), v) {}
    int size() const { return (int)m_v.size(); }
    int count() const { return (int)m_v.size(); }
    bool isEmpty() const { return m_v.empty(); }
    T& operator[](int i) { return m_v[(size_t)i]; }
    const T& operator[](int i) const { return m_v[(size_t)i]; }
    const T& at(int i) const { return m_v.at((size_t)i); }
    void push_back(const T& v) { m_v.push_back(v); }
    void append(const T& v) { m_v.push_back(v); }
    QVector& operator<<(const T& v) { m_v.push_back(v); return *this; }
    void fill(const T& v, int n = -1) {
        if (n >= 0) m_v.assign((size_t)n, v);
        else std::fill(m_v.begin(), m_v.end(), v);
    }
    void resize(int n) { m_v.resize((size_t)std::max(n, 0)); }
    void clear() { m_v.clear(); }
    bool contains(const T& v) const { return std::find(m_v.begin(), m_v.end(), v) != m_v.end(); }
    int indexOf(const T& v) const {
        auto it = std::find(m_v.begin(), m_v.end(), v);
        return it == m_v.end() ? -1 : (int)(it - m_v.begin());
    }
    T* data() { return m_v.data(); }
    typename std::vector<T>::iterator begin() { return m_v.begin(); }
    typename std::vector<T>::iterator end() { return m_v.end(); }
    typename std::vector<T>::const_iterator begin() const { return m_v.begin(); }
    typename std::vector<T>::const_iterator end() const { return m_v.end(); }

private:
    std::vector<T> m_v;
};

template <class T>
class QList {
public:
    QList() {}
    int size() const { return (int)m_v.size(); }
    int count() const { return (int)m_v.size(); }
    int count(const T& v) const { return (int)std::count(m_v.begin(), m_v.end(), v); }
    int length() const { return (int)m_v.size(); }
    bool isEmpty() const { return m_v.empty(); }
    bool empty() const { return m_v.empty(); }
    void reserve(int n) { m_v.reserve((size_t)std::max(n, 0)); }
    T& operator[](int i) { return m_v[(size_t)i]; }
    const T& operator[](int i) const { return m_v[(size_t)i]; }
    const T& at(int i) const { return m_v.at((size_t)i); }
    T& first() { return m_v.front(); }
    T& last() { return m_v.back(); }
    void push_back(const T& v) { m_v.push_back(v); }
    void append(const T& v) { m_v.push_back(v); }
    void prepend(const T& v) { m_v.insert(m_v.begin(), v); }
    QList& operator<<(const T& v) { m_v.push_back(v); return *this; }
    void removeAt(int i) { m_v.erase(m_v.begin() + i); }
    T takeAt(int i) { T v = m_v[(size_t)i]; removeAt(i); return v; }
    bool removeOne(const T& v) {
        auto it = std::find(m_v.begin(), m_v.end(), v);
        if (it == m_v.end()) return false;
        m_v.erase(it);
        return true;
    }
    void clear() { m_v.clear(); }
    bool contains(const T& v) const { return std::find(m_v.begin(), m_v.end(), v) != m_v.end(); }
    int indexOf(const T& v) const {
        auto it = std::find(m_v.begin(), m_v.end(), v);
        return it == m_v.end() ? -1 : (int)(it - m_v.begin());
    }
    typename std::vector<T>::iterator begin() { return m_v.begin(); }
    typename std::vector<T>::iterator end() { return m_v.end(); }
    typename std::vector<T>::const_iterator begin() const { return m_v.begin(); }
    typename std::vector<T>::const_iterator end() const { return m_v.end(); }

private:
    std::vector<T> m_v;
};

class QStringList : public QList<QString> {
public:
    QStringList& operator<<(const QString& s) { push_back(s); return *this; }
};

class QObject {
public:
    explicit QObject(QObject* parent = nullptr) { (void)parent; }
    virtual ~QObject() {}
    void setObjectName(const QString& n) { m_name = n; }
    QString objectName() const { return m_name; }

private:
    QString m_name;
};

// Text and binary streams: the compiled files write names and diagnostics
// through them; the text stream keeps what it is given in its string.
class QTextStream {
public:
    enum Status { Ok, ReadPastEnd, ReadCorruptData };
    Status status() const { return Ok; }
    QTextStream() {}
    explicit QTextStream(QString* s) : m_target(s) {}
    template <class T>
    QTextStream& operator<<(const T& v) {
        m_buf << v;
        return *this;
    }
    template <class T>
    QTextStream& operator>>(T&) { return *this; }
    void flush() {
        if (m_target) *m_target = QString(m_target->toStdString() + m_buf.str());
        m_buf.str("");
    }
    ~QTextStream() { flush(); }

private:
    QString* m_target = nullptr;
    std::ostringstream m_buf;
};
// The binary stream only carries the random-number state in the reference's
// checkpoints, which the harness never writes.
class QDataStream {
public:
    enum Status { Ok, ReadPastEnd, ReadCorruptData };
    Status status() const { return Ok; }
    template <class T>
    QDataStream& operator<<(const T&) { return *this; }
    template <class T>
    QDataStream& operator>>(T&) { return *this; }
};

class QDebug {
public:
    template <class T>
    QDebug& operator<<(const T&) { return *this; }
};
inline QDebug qDebug() { return QDebug(); }
inline void qDebug(const char*, ...) {}
inline QDebug qWarning() { return QDebug(); }
inline void qWarning(const char*, ...) {}
// qFatal: the reference aborts; here the harness catches the error and reports it
[[noreturn]] inline void qFatal(const char* fmt, ...) {
    char b[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(b, sizeof b, fmt, ap);
    va_end(ap);
    throw std::runtime_error(b);
}

template <class T>
inline const T& qMin(const T& a, const T& b) { return std::min(a, b); }
template <class T>
inline const T& qMax(const T& a, const T& b) { return std::max(a, b); }
template <class It>
inline void qSort(It a, It b) { std::sort(a, b); }
template <class C>
inline void qSort(C& c) { std::sort(c.begin(), c.end()); }

class QDateTime {
public:
    static QDateTime currentDateTime() { return QDateTime(); }
};
class QVariant {
public:
    QVariant() {}
    template <class T>
    QVariant(const T&) {}
};
class QThread {
public:
    static int idealThreadCount() { return 1; }
};
class QThreadPool {
public:
    static QThreadPool* globalInstance() {
        static QThreadPool p;
        return &p;
    }
    int maxThreadCount() const { return m_n; }
    void setMaxThreadCount(int n) { m_n = n; }

private:
    int m_n = 1;
};
class QFileInfo {};
class QDir {};
